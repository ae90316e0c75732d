// plan_enum_rrs.cpp -- PlanEnumRRS (include/fmcs/plan_enum_rrs.h).
// Reference: src/plan_enum_rrs.cpp:7-396 (random samples, neighbours, cost
// from per-column statistics, time-limited stop).
#include "../../../include/fmcs/plan_enum_rrs.h"

#include <algorithm>
#include <cmath>

namespace multiAttrSort {

PlanEnumRRS::PlanEnumRRS(uint64_t num_rows, uint32_t col_width_sum, uint32_t max_round,
                         std::vector<uint32_t> column_order, uint32_t num_columns, std::vector<uint32_t> bw,
                         std::vector<uint32_t> base_col_card, double time_limit)
    : RRS<std::vector<uint32_t>, double>(0.99, 0.1, 0.99, 0.8, 0.5, 0.001), num_rows_(num_rows),
      col_width_sum_(col_width_sum), max_round_(std::max<uint32_t>(1, max_round)), columnOrder_(column_order),
      num_columns_(num_columns), bw_(bw), base_col_card_(base_col_card), time_limit_(time_limit),
      start_(std::chrono::steady_clock::now()), tables_(GpuCostTables::Cached()), rng_(0xF17C0001ull)
{
}

double PlanEnumRRS::group_num(uint32_t bits) const
{
    double g = 1.0;
    for (uint32_t i = 0; i < num_columns_ && bits > 0; ++i) {
        const uint32_t c = columnOrder_[i];
        const uint32_t take = std::min(bits, bw_[c]);
        g *= std::pow(std::pow((double)std::max<uint32_t>(1, base_col_card_[c]), 1.0 / bw_[c]), (double)take);
        bits -= take;
    }
    return std::min(g, (double)num_rows_);
}

PlanEnumRRS::PointType PlanEnumRRS::GetRandomSample()
{
    // random number of rounds that can hold the width, then random cuts
    const uint32_t min_rounds = (col_width_sum_ + 63) / 64;
    const uint32_t hi = std::max(min_rounds, std::min(max_round_, col_width_sum_));
    std::uniform_int_distribution<uint32_t> rd(min_rounds, hi);
    for (;;) {
        const uint32_t rounds = rd(rng_);
        std::vector<uint32_t> cuts;
        std::uniform_int_distribution<uint32_t> cd(1, col_width_sum_ - 1);
        while (cuts.size() + 1 < rounds) {
            uint32_t c = cd(rng_);
            if (std::find(cuts.begin(), cuts.end(), c) == cuts.end()) cuts.push_back(c);
        }
        std::sort(cuts.begin(), cuts.end());
        PointType p;
        uint32_t prev = 0;
        for (uint32_t c : cuts) {
            p.push_back(c - prev);
            prev = c;
        }
        p.push_back(col_width_sum_ - prev);
        bool ok = true;
        for (uint32_t w : p) ok = ok && w >= 1 && w <= 64;
        if (ok) return p;
    }
}

PlanEnumRRS::CostType PlanEnumRRS::GetCost(const PointType &split)
{
    ++counter_;
    searchedPlans.insert(split);
    double ms = 0.0;
    uint32_t prefix = 0;
    for (size_t r = 0; r < split.size(); ++r) {
        const uint32_t w = split[r];
        const uint32_t B = w <= 16 ? 2 : (w <= 32 ? 4 : 8);
        const int b = GpuCostTables::BankIndex(B);
        if (r > 0) ms += tables_.gather[b] * num_rows_ / 1e6;
        const double groups = r == 0 ? 1.0 : group_num(prefix);
        ms += tables_.SortRoundMs(num_rows_, (double)num_rows_ / groups, B, w);
        ms += tables_.boundary[b] * num_rows_ / 1e6 + tables_.round_fixed_ms;
        ms += tables_.stitch_per_byte * 2.0 * B * num_rows_ / 1e6;
        prefix += w;
    }
    return ms;
}

bool PlanEnumRRS::StopCritera()
{
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start_).count();
    return ms > time_limit_;
}

PlanEnumRRS::PointType PlanEnumRRS::GetRandomNeighbor(const PointType &point, double ro)
{
    // move up to ro * total bits across one boundary between adjacent banks
    if (point.size() < 2) return GetRandomSample();
    const uint32_t maxmove = std::max<uint32_t>(1, (uint32_t)std::ceil(ro * col_width_sum_));
    std::uniform_int_distribution<size_t> bd(0, point.size() - 2);
    std::uniform_int_distribution<int> md(-(int)maxmove, (int)maxmove);
    for (int tries = 0; tries < 64; ++tries) {
        PointType p = point;
        const size_t i = bd(rng_);
        const int m = md(rng_);
        const int a = (int)p[i] - m, c = (int)p[i + 1] + m;
        if (m == 0 || a < 1 || c < 1 || a > 64 || c > 64) continue;
        p[i] = (uint32_t)a;
        p[i + 1] = (uint32_t)c;
        return p;
    }
    return point;
}

}  // namespace multiAttrSort
