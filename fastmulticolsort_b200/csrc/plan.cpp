// plan.cpp -- slice records of a massaging plan (see plan.h).
#include "plan.h"

namespace fmcs {

uint32_t bank_bytes_for(uint32_t bits, bool hash_path)
{
    if (hash_path && bits <= 8) return 1;
    if (bits <= 16) return 2;
    if (bits <= 32) return 4;
    return 8;
}

bool build_plan(const uint32_t *bw, uint32_t ncols, const uint32_t *col_order, const uint32_t *split,
                uint32_t nbanks, bool hash_path, Plan &out, std::string &err)
{
    out.banks.clear();
    if (ncols == 0 || nbanks == 0) {
        err = "empty plan";
        return false;
    }
    uint64_t total_old = 0, total_new = 0;
    std::vector<bool> seen(ncols, false);
    for (uint32_t c = 0; c < ncols; ++c) {
        if (col_order[c] >= ncols || seen[col_order[c]]) {
            err = "column order is not a permutation";
            return false;
        }
        seen[col_order[c]] = true;
        if (bw[c] == 0 || bw[c] > 64) {
            err = "column width outside 1..64";
            return false;
        }
        total_old += bw[c];
    }
    for (uint32_t b = 0; b < nbanks; ++b) {
        if (split[b] == 0 || split[b] > 64) {
            err = "split entry outside 1..64";
            return false;
        }
        total_new += split[b];
    }
    if (total_old != total_new) {
        err = "split does not add up to the column widths";
        return false;
    }
    out.banks.resize(nbanks);
    for (uint32_t b = 0; b < nbanks; ++b) {
        out.banks[b].bits = split[b];
        out.banks[b].bytes = bank_bytes_for(split[b], hash_path);
    }
    // Walk old columns (in col_order) and new banks together; every step takes
    // min(bits left in the column, bits left in the bank).
    uint32_t oc = 0, nb = 0, start = 1;
    uint32_t old_left = bw[col_order[0]], new_left = split[0];
    while (nb < nbanks) {
        const uint32_t take = old_left < new_left ? old_left : new_left;
        out.banks[nb].slices.push_back(SliceRec{col_order[oc], start, start + take - 1});
        start += take;
        old_left -= take;
        new_left -= take;
        if (old_left == 0) {
            ++oc;
            if (oc < ncols) old_left = bw[col_order[oc]];
            start = 1;
        }
        if (new_left == 0) {
            ++nb;
            if (nb < nbanks) new_left = split[nb];
        }
    }
    return true;
}

}  // namespace fmcs
