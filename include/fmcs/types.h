// fmcs/types.h -- the reference's public data types, kept name-for-name so that
// code written against FastMultiColSort compiles against this library.
//
// Reference: src/types.h (construct_entry_t :42-46, compose_params_t :169-186,
// group_info_t :188-195, setting_t :198-236, enums :116-166) and
// src/params.h:9-13 (surrogate_t).  Timing fields keep their names; here they
// hold MILLISECONDS measured with CUDA events / steady_clock (the reference
// stores rdtsc cycles).
#pragma once

#include <cstdint>
#include <string>

#if defined(__GNUC__)
#define FMCS_CXX_API __attribute__((visibility("default")))
#else
#define FMCS_CXX_API
#endif

namespace multiAttrSort {

#ifdef OID_WIDTH_8B
#error "the B200 path uses 32-bit row ids (n < 2^32)"
#endif
typedef uint32_t surrogate_t;

/** One slice of an original column that goes into a massaged bank:
 *  bits [start, end], 1-based from the MSB of the column's declared width. */
struct construct_entry_t {
    uint32_t finalIdx;
    uint32_t start;
    uint32_t end;
};

enum class IntrinsicsType { AVX, SSE, SCALAR };
enum class Baseline { aligned32, adaptive };
enum class SortAlgo { mergesort, radixsort };
enum class PackOIDType { pack, nonpack };
enum class ComposerType { chaining, stitching };

struct dataset_t {
    uint64_t nrows;
    uint32_t ncolumns;
    std::string column_bitwidth;
    uint32_t zipf;
    uint32_t cardinality;
    uint32_t group_num = 2;
};

struct compose_params_t {
    SortAlgo sortalgo = SortAlgo::radixsort;   // the GPU path always radix-sorts
    PackOIDType packtype = PackOIDType::nonpack;
    bool is_oid_encoded = false;
    bool *column_asc_desc = nullptr;   // parsed but, as in the reference, every column sorts ascending
    uint32_t *bitwidth = nullptr;      // declared bit width of each column
    Baseline baseline = Baseline::adaptive;
    uint32_t colwidth_sum = 0;         // sum of bitwidth[]
    uint32_t ordered = 1;              // 0: GROUP BY (column order may be permuted)
    uint32_t hash_type = 1;            // 1 reordered, 2 partitioned-reordered, 0 non-reordered
};

struct group_info_t {
    uint32_t ngroups = 0;            // groups (segments) sorted in the last round
    uint32_t sum_group_size = 0;
    uint32_t ngroups_incache = 0;    // segments sorted on chip (<= 4096 rows)
    uint32_t ngroups_outofcache = 0; // segments sorted through HBM radix levels
    uint32_t ngroups_gtOne = 0;
};

struct setting_t {
    uint32_t nthreads = 1;
    IntrinsicsType intrinType = IntrinsicsType::AVX;
    uint32_t bitwidth = 0;
    /* milliseconds of the last run, per stage */
    double time_tupleReconstruct = 0.0;   // gathers (BATproject)
    double time_orderGroupInfo = 0.0;     // group ids
    double time_multipass_sort = 0.0;     // all sort rounds
    double time_firstpass_sort = 0.0;     // round 0
    double time_mmcpyOrderGroup = 0.0;
    double time_extractGrop = 0.0;
    double time_stitching = 0.0;
    double time_optimization = 0.0;
    double time_hashReordering = 0.0;
    uint32_t partition_fanout = 1;
};

}  // namespace multiAttrSort
