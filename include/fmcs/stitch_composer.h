// fmcs/stitch_composer.h -- StitchComposer: code massaging (bit stitching and
// bit borrowing) with a cost-model plan search, on the GPU.
//
// Reference: src/stitch_composer.h:13-250 / src/stitch_composer.cpp; same
// class name, constructor and entry points (RunAnInstance, TwoRoundsExhaustive,
// ExhaustiveSearch, SortAllColumns_Nonpack -> optimizeAndRun, HashAllColumns,
// RunAnInstance_hash, TwoRoundsExhaustive_hash, CostModelComparison,
// run_single_plan, run_single_plan_hash).  run_single_plan does not hard-code a
// CPU ChainComposer (src/stitch_composer.cpp:745): it runs the whole plan --
// fused stitch of every bank, then the sort rounds -- through fmcs_run_plan.
// Reported times are milliseconds (the reference prints cycles per row).
#pragma once

#include <cstdint>
#include <set>
#include <string>
#include <vector>

#include "composer.h"
#include "cost_model.h"

namespace multiAttrSort {

class FMCS_CXX_API StitchComposer : public Composer {
  public:
    StitchComposer(setting_t setting, uint32_t ncolumns, uint64_t nrows, compose_params_t params,
                   Column **column_values);
    ~StitchComposer() override {}

    // ---- cost model (static, like the reference's estimate_* functions);
    // values are estimated GPU milliseconds
    static double estimate_mergesort_uint16(double nitems);
    static double estimate_mergesort_uint32(double nitems);
    static double estimate_mergesort_uint64(double nitems);
    /** assembleStatistics[from][to] / shiftStatistics[to], bank classes 16/32/64
     *  (src/stitch_composer.cpp:288-378 builds them). */
    static double estimate_stitch(uint32_t assembleStatistics[][3], uint32_t shiftStatistics[], uint32_t nitems);
    static double estimate_tuple_reconstruct(const uint32_t *bytewidths, const uint32_t column_num,
                                             const uint64_t rows_num);

    void SortAllColumns_Pack() override {}
    /** Baseline (one round per column) then optimizeAndRun(). */
    void SortAllColumns_Nonpack() override;
    /** Every split of the first two columns into one or two banks, run and timed. */
    void ExhaustiveSearch() override;
    /** Bit-borrowing sweep [w0 - s, w1 + s] for s in [-w1, w0]
     *  (src/stitch_composer.cpp:4197-4258); prints s, round-0 ms, other rounds ms, other ms. */
    void TwoRoundsExhaustive() override;
    /** Baseline [w0, w1] and the given plan, e.g. "50" or "6B44"
     *  (src/stitch_composer.cpp:4051-4120). */
    void RunAnInstance(std::string instance) override;
    /** Estimated versus measured cost of the enumerated plans
     *  (src/stitch_composer.cpp:4337-4469). */
    void CostModelComparison() override;
    void RunAnInstance_hash(std::string instance) override;
    void TwoRoundsExhaustive_hash() override;
    /** Hash grouping with the optimizer's plan. */
    void HashAllColumns() override;

    /** Run one plan: stitch banks per `curSplit` over the columns in
     *  `columnOrder`, then one sort round per bank.  breakdown[0..5] =
     *  {stitch, gathers, group ids, all sort rounds, round 0, group ids} in ms
     *  (the reference's breakdown slots, src/stitch_composer.cpp:719, 755-767).
     *  Returns the total ms.  The result is kept (GetOrder/GetGroup). */
    double run_single_plan(uint32_t *columnOrder, std::vector<uint32_t> &curSplit, double *breakdown);
    double run_single_plan_hash(uint32_t *columnOrder, std::vector<uint32_t> &curSplit, double *breakdown);

    /** The optimizer alone: best plan and column order under the cost model
     *  (src/stitch_composer.cpp:3839-3984 without the final run). */
    std::vector<uint32_t> OptimizePlan(std::vector<uint32_t> *columnOrder = nullptr, double *est_ms = nullptr);
    /** Estimated ms of one plan. */
    double EstimatePlan(const uint32_t *columnOrder, const std::vector<uint32_t> &split);
    /** Estimated number of distinct values of the first `bit_position` bits of
     *  the stitched key (src/stitch_composer.cpp:1845-1867). */
    double estimateGroupNum(const uint32_t bit_position, const uint32_t *columnOrder);

    /** All splits of `n` bits into exactly round_num banks of <= maxValue bits
     *  (src/stitch_composer.cpp:205-230). */
    void split_exhaustive_certain_round(int n, int curRound, const int round_num, const int maxValue,
                                        std::vector<std::vector<uint32_t>> &split_enum);
    /** Greedy plans with round_num > 2 rounds: per bank-size category, each
     *  round's cut chosen by the cost of the next round
     *  (src/stitch_composer.cpp:1991-2125). */
    void find_greedy_plans(uint32_t round_num, std::vector<std::vector<uint32_t>> &validPlans,
                           const uint32_t *columnOrder);
    /** Sorting cost of one round given its average group size and bank class
     *  (0: 16-bit, 1: 32-bit, 2: 64-bit), src/stitch_composer.cpp:2186-2226. */
    double calculate_single_column_cost(const double groupsz, const uint32_t banksz_type);

    const GpuCostTables &Tables() const { return tables_; }
    void SetTables(const GpuCostTables &t) { tables_ = t; }

    std::vector<uint64_t> base_col_card;
    std::vector<double> card_per_bit;
    double shrink_factor = 1.0;

  protected:
    void optimizeAndRun();
    void permutations(std::vector<uint32_t> &arr, uint32_t k, std::vector<std::vector<uint32_t>> &out);
    double run_plan(const uint32_t *columnOrder, const std::vector<uint32_t> &split, bool hash, double *breakdown);
    static std::vector<uint32_t> parse_plan(const std::string &instance);

    GpuCostTables tables_;
    uint32_t partitions_[64] = {};
};

}  // namespace multiAttrSort
