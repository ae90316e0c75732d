// plan.h -- massaging plans: the slice records of each bank and the bank width.
//
// Reference: construct_entry_t (src/types.h:42-46) and the record builder of
// StitchComposer::run_single_plan (src/stitch_composer.cpp:568-612); bank
// widths per src/stitch_composer.cpp:622-650 (sort: 2/4/8 bytes) and
// :879-912 (hash: also 1 byte).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fmcs {

constexpr uint32_t kMaxPlanCols = 64;
constexpr uint32_t kMaxPlanBanks = 64;

struct SliceRec {
    uint32_t col;    // source column index (already mapped through the column order)
    uint32_t start;  // 1-based from the MSB of the declared width
    uint32_t end;    // inclusive
};

struct BankPlan {
    uint32_t bits = 0;   // split entry
    uint32_t bytes = 0;  // storage width
    std::vector<SliceRec> slices;
};

struct Plan {
    std::vector<BankPlan> banks;
};

uint32_t bank_bytes_for(uint32_t bits, bool hash_path);

// Builds the plan; false (with a message) when the split does not add up to the
// columns' widths or a split entry is outside 1..64.
bool build_plan(const uint32_t *bw, uint32_t ncols, const uint32_t *col_order, const uint32_t *split,
                uint32_t nbanks, bool hash_path, Plan &out, std::string &err);

}  // namespace fmcs
