// fmcs/plan_enum_rrs.h -- massaging-plan enumeration by Recursive Random
// Search (reference: src/plan_enum_rrs.h:17-83, same class and constructor).
// A point is a split (bank widths in bits, each 1..64, summing to the total
// width); its cost is the GPU cost model's estimate (GpuCostTables).
#pragma once

#include <chrono>
#include <cstdint>
#include <set>
#include <vector>

#include "cost_model.h"
#include "rrs.h"

namespace multiAttrSort {

class FMCS_CXX_API PlanEnumRRS : public RRS<std::vector<uint32_t>, double> {
  public:
    typedef std::vector<uint32_t> PointType;
    typedef double CostType;

    /** time_limit in milliseconds of search. */
    PlanEnumRRS(uint64_t num_rows, uint32_t col_width_sum, uint32_t max_round, std::vector<uint32_t> column_order,
                uint32_t num_columns, std::vector<uint32_t> bw, std::vector<uint32_t> base_col_card,
                double time_limit);

    PointType GetRandomSample() override;
    CostType GetCost(const PointType &point) override;
    bool StopCritera() override;
    PointType GetRandomNeighbor(const PointType &point, double ro) override;

    std::set<std::vector<uint32_t>> ObtainPlans() { return searchedPlans; }
    void SetTables(const GpuCostTables &t) { tables_ = t; }

  protected:
    size_t counter_ = 0;
    const uint64_t num_rows_;
    const uint32_t col_width_sum_;
    const uint32_t max_round_;
    const std::vector<uint32_t> columnOrder_;
    const uint32_t num_columns_;
    const std::vector<uint32_t> bw_;
    const std::vector<uint32_t> base_col_card_;
    const double time_limit_;
    std::set<std::vector<uint32_t>> searchedPlans;
    std::chrono::steady_clock::time_point start_;
    GpuCostTables tables_;
    std::mt19937_64 rng_;

  private:
    double group_num(uint32_t bits) const;
};

}  // namespace multiAttrSort
