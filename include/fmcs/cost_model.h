// fmcs/cost_model.h -- the cost model of massaging plans, for the GPU path.
//
// Reference: the cost functions of StitchComposer (estimate_mergesort_uint{16,
// 32,64}, src/stitch_composer.cpp:3447-3496; estimate_stitch, :2850-2889;
// estimate_tuple_reconstruct, :2813-2848; calculate_single_column_cost,
// :2186-2226) with cycle tables calibrated on one Haswell core
// (src/params.h:200-2283).  The structure is kept -- a plan costs its stitch,
// its gathers, its group-id scans and one sort per round, each sort costed from
// the round's AVERAGE group size, which comes from per-column cardinalities --
// but every table is in milliseconds per million rows measured on the GPU, per
// bank width (2, 4, 8 bytes), and the sort cost follows the GPU engine: a
// group of g rows is sorted on chip if g <= local_max (8192 unless tuned;
// cost by log2 g), else after ceil(log256(g / local_max)) HBM radix levels.  The autotuner
// (fastmulticolsort_b200/autotune.py) re-measures the tables and writes them
// as JSON; GpuCostTables::Load reads them back.
#pragma once

#include <cstdint>
#include <string>

#include "types.h"

namespace multiAttrSort {

struct FMCS_CXX_API GpuCostTables {
    // all costs: milliseconds per million rows; index b: 0 = 2-byte bank,
    // 1 = 4-byte, 2 = 8-byte
    double stitch_per_byte = 0.00021;   // per byte moved (sources read + bank written)
    double gather[3] = {0.0035, 0.0040, 0.0055};
    double boundary[3] = {0.0030, 0.0040, 0.0060};
    double msd_level[3] = {0.010, 0.013, 0.018};   // one HBM radix level over the rows of large groups
    // on-chip sort of groups of ~2^k rows, k = 0..13
    static constexpr int kLocalSizes = 14;
    double local[3][kLocalSizes] = {
        {0.0, 0.004, 0.004, 0.004, 0.005, 0.006, 0.007, 0.008, 0.009, 0.011, 0.013, 0.015, 0.018, 0.020},
        {0.0, 0.004, 0.004, 0.005, 0.006, 0.007, 0.008, 0.010, 0.011, 0.013, 0.015, 0.018, 0.021, 0.024},
        {0.0, 0.005, 0.005, 0.006, 0.007, 0.008, 0.010, 0.012, 0.014, 0.016, 0.019, 0.023, 0.028, 0.032}};
    double round_fixed_ms = 0.03;   // per-round launch and synchronization overhead
    uint32_t local_max = 8192;      // largest group sorted on chip (the engine's knob)

    static int BankIndex(uint32_t bank_bytes) { return bank_bytes <= 2 ? 0 : (bank_bytes <= 4 ? 1 : 2); }
    /** Read a table written by the autotuner (JSON); false if absent/invalid. */
    bool Load(const std::string &path);
    /** The tables of the autotuner's last run next to libfmcs.so
     *  (tuning/b200.json), or FMCS_TUNING, or the built-in defaults, read
     *  from the file on every call. */
    static GpuCostTables Default();
    /** Default() read once per process (on the first call) and kept: the
     *  tables the composers and the static estimate_* functions use. */
    static const GpuCostTables &Cached();

    /** Estimated ms to sort ONE group of g rows of the given bank width. */
    double SortGroupMs(double g, uint32_t bank_bytes, uint32_t key_bits) const;
    /** Estimated ms of one sort round over n rows in groups of average size g. */
    double SortRoundMs(uint64_t n, double g, uint32_t bank_bytes, uint32_t key_bits) const;
    /** The same with the key's distribution: split[l] = distinct values of
     *  the top 8 * (l + 1) key bits inside a group (a radix level cannot split
     *  a group into more parts than that), for l < nsplit. */
    double SortGroupMs(double g, uint32_t bank_bytes, uint32_t key_bits, const double *split, int nsplit) const;
    double SortRoundMs(uint64_t n, double g, uint32_t bank_bytes, uint32_t key_bits, const double *split,
                       int nsplit) const;
};

}  // namespace multiAttrSort
