// fmcs/composer.h -- Composer and ChainComposer: the round engine of the
// multi-column sort, on the GPU.
//
// Reference: src/composer.h:15-177 and src/chain_composer.h:14-40; same class
// names, constructor and methods, so that driver code that builds
// Column**, setting_t and compose_params_t and calls SortAllColumns() /
// HashAllColumns() works unchanged.  Differences, all deliberate:
//   - every round runs on the GPU through the C ABI (fmcs_sort_round,
//     fmcs_hash_round, fmcs_hash_round_unordered);
//   - results are kept, not freed (the reference frees them inside
//     multiRoundSorting, src/composer.cpp:132-134): GetOrder(), GetGroup(),
//     GetGroupCount(), CopyOrderTo(), CopyGroupTo();
//   - the sort is stable: ties keep ascending oid (the reference's AVX merge
//     sort leaves them in arbitrary order);
//   - the last round's group ids are computed too (the reference skips them).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "column.h"
#include "types.h"

namespace multiAttrSort {

class FMCS_CXX_API Composer {
  public:
    Composer(setting_t setting, uint32_t ncolumns, uint64_t nrows, compose_params_t params, Column **column_values);
    Composer();
    virtual ~Composer();

    /** Sort by all columns in order (ORDER BY); dispatches on packtype like
     *  the reference (only the non-packed layout exists). */
    void SortAllColumns();

    setting_t getSetting() { return setting_; }
    group_info_t getGroupInfo() { return group_info_; }

    /** Use this context instead of the per-thread default. */
    void SetContext(fmcs_ctx *ctx) { ctx_ = ctx; }
    fmcs_ctx *GetContext();

    /** Results of the last SortAllColumns()/HashAllColumns(): the oid
     *  permutation and the dense group id of every output position. */
    std::vector<surrogate_t> GetOrder() const;
    std::vector<surrogate_t> GetGroup() const;
    uint32_t GetGroupCount() const { return ngroups_; }
    /** Copy the results into caller memory (host or device). */
    void CopyOrderTo(surrogate_t *dst) const;
    void CopyGroupTo(surrogate_t *dst) const;
    /** Device pointers of the results (valid until the next run). */
    const surrogate_t *DeviceOrder() const { return d_order_; }
    const surrogate_t *DeviceGroup() const { return d_group_[final_group_]; }

    // ---- members public as in the reference (its `//protected:` at composer.h:50)
    uint32_t num_columns_;
    uint64_t num_rows_;
    Column **column_values_;
    setting_t setting_;
    compose_params_t compose_params_;
    group_info_t group_info_;

    virtual void SortAllColumns_Pack() = 0;
    virtual void SortAllColumns_Nonpack() = 0;
    virtual void ExhaustiveSearch() = 0;
    virtual void TwoRoundsExhaustive() = 0;
    virtual void RunAnInstance(std::string intance) = 0;
    virtual void CostModelComparison() = 0;
    virtual void RunAnInstance_hash(std::string intance) = 0;
    virtual void TwoRoundsExhaustive_hash() = 0;
    virtual void HashAllColumns() = 0;

    /** One sort round per column (src/composer.cpp:48-135). */
    void multiRoundSorting();
    /** Hash grouping rounds, re-clustering between rounds
     *  (src/composer.cpp:137-227). */
    void multiRoundHashing_reordered();
    /** Same result as multiRoundHashing_reordered (the reference's partitioned
     *  variant differs only in how it walks memory). */
    void multiRoundHashing_partitioned_reordered();
    /** Group ids by first appearance of the column-prefix tuple in ROW order,
     *  no re-clustering (src/composer.cpp:321-381). */
    void multiRoundHashing_non_reordered();

    /** One sort round, the reference's sortByGroup<T> (src/composer.cpp:1222-1408):
     *  inGroup == NULL sorts inValues IN PLACE with the oids in `order`
     *  (round 0, order = iota); otherwise sorts inValues[order[i]] inside every
     *  run of equal inGroup.  outGroup receives the group ids unless
     *  isLastRound.  Pointers may be host or device memory. */
    template <class T>
    void sortByGroup(surrogate_t *outGroup, T *inValues, surrogate_t *order, surrogate_t *inGroup, bool asc_desc,
                     uint32_t bitwidth, bool isLastRound)
    {
        (void)asc_desc;   // every column sorts ascending, as in the reference
        sort_round_any(outGroup, inValues, sizeof(T), order, inGroup, bitwidth, isLastRound);
    }

    /** values_reordered[i] = values[order[i]] into a new device buffer that the
     *  caller frees with cudaFree (Composer::BATproject, src/composer.cpp:608-628). */
    template <class T>
    T *BATproject(const T *values, const surrogate_t *order)
    {
        return (T *)gather_any(values, sizeof(T), order);
    }

  protected:
    void sort_round_any(surrogate_t *outGroup, void *inValues, uint32_t bytes, surrogate_t *order,
                        surrogate_t *inGroup, uint32_t bitwidth, bool isLastRound);
    void *gather_any(const void *values, uint32_t bytes, const surrogate_t *order);
    void ensure_buffers();
    void hash_rounds(bool reordered);

    fmcs_ctx *ctx_ = nullptr;
    surrogate_t *d_order_ = nullptr;
    surrogate_t *d_group_[2] = {nullptr, nullptr};
    uint64_t buf_rows_ = 0;
    int final_group_ = 0;
    uint32_t ngroups_ = 0;
};

class FMCS_CXX_API ChainComposer : public Composer {
  public:
    ChainComposer(setting_t setting, uint32_t ncolumns, uint64_t nrows, compose_params_t params,
                  Column **column_values)
        : Composer(setting, ncolumns, nrows, params, column_values)
    {
    }
    ChainComposer() {}
    ~ChainComposer() override {}

    void SortAllColumns_Pack() override {}
    void SortAllColumns_Nonpack() override { multiRoundSorting(); }
    void ExhaustiveSearch() override {}
    void TwoRoundsExhaustive() override {}
    void RunAnInstance(std::string) override {}
    void CostModelComparison() override {}
    void RunAnInstance_hash(std::string) override {}
    void TwoRoundsExhaustive_hash() override {}
    /** hash_type 1 (reordered) / 2 (partitioned) / 0 (non-reordered),
     *  src/chain_composer.cpp:16-25. */
    void HashAllColumns() override;
};

}  // namespace multiAttrSort
