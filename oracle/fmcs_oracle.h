/*
 * fmcs_oracle.h -- CPU restatement of FastMultiColSort's multi-column sort
 * path, used ONLY as the parity oracle of the CUDA path (tests, the smoke check and
 * the CPU-baseline leg of the benchmark).  Nothing in the shipped library
 * links or calls this code.
 *
 * Parity is pinned two ways (see tests/test_oracle.py):
 *   - against the reference's own composer, compiled from its sources by
 *     oracle/Makefile into oracle/_ref/ and driven by oracle/ref_harness.cpp;
 *   - against fixtures in tests/golden/ produced by that harness
 *     (tests/golden/make_golden.py) plus the 9-tuple known-answer case of the
 *     reference's tests/subgroup_test.cpp:98-145.
 *
 * Conventions (reference: src/params.h:9-13, src/types.h:42-46):
 *   oid / order / group are uint32; banks are uint8/16/32/64.
 *   The reference's sort is not stable; the oracle is stable, which equals
 *   the reference's output once ties are canonicalised to ascending oid.
 */
#ifndef FMCS_ORACLE_H
#define FMCS_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One slice of a source column that goes into a bank.  Bits are numbered
 * 1-based from the MSB of the source's DECLARED width `src_bits`
 * (reference: src/stitch_composer.cpp:568-612, src/column.h:208-1060). */
typedef struct {
    const void *src;
    uint32_t src_bytes;   /* 1, 2, 4 or 8 */
    uint32_t src_bits;    /* declared width of the source column */
    uint32_t start;       /* first bit, 1-based from the MSB */
    uint32_t end;         /* last bit, inclusive */
} orc_slice;

/* construct_entry_t (reference: src/types.h:42-46). */
typedef struct {
    uint32_t final_idx;
    uint32_t start;
    uint32_t end;
} orc_record;

/* Record builder of run_single_plan (src/stitch_composer.cpp:568-612).
 * rec must hold ncols+nbanks entries; nrec[b] receives the count of bank b;
 * records of bank b are stored consecutively after those of bank b-1.
 * Returns the total record count or -1 when the split does not add up. */
int orc_plan_records(const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                     const uint32_t *split, uint32_t nbanks,
                     orc_record *rec, uint32_t *nrec);

/* Bank width chosen for a split entry: sort path 2/4/8 bytes
 * (src/stitch_composer.cpp:622-650), hash path also 1 byte (:879-912). */
uint32_t orc_bank_bytes(uint32_t bits, int hash_path);

/* ShiftLeftBatch + AssembleFromColumn for every slice of one bank
 * (src/column.h:105-180, 208-1060). */
int orc_stitch(const orc_slice *slices, uint32_t nslices,
               void *bank, uint32_t bank_bytes, uint64_t n);

/* One sort round, Composer::sortByGroup<T> (src/composer.cpp:1222-1408):
 *   in_group == NULL: round 0, order := stable argsort of bank (order is
 *                     output only; the reference starts from iota,
 *                     src/composer.cpp:60-63);
 *   otherwise:        values := bank[order[i]] (BATproject, :608-628), then a
 *                     stable sort inside every run of equal in_group (:1280-1335),
 *                     order permuted alongside.
 * out_group (may be NULL = last round) gets extractGroupInfo (:630-678).
 * sorted_keys (may be NULL) receives the sorted bank values.
 * *ngroups receives the number of groups (max id + 1), 0 when out_group is NULL. */
int orc_sort_round(const void *bank, uint32_t bank_bytes, uint32_t *order,
                   const uint32_t *in_group, uint32_t *out_group,
                   void *sorted_keys, uint64_t n, uint32_t *ngroups);

/* One hash round, Composer::hashByGroup_reordered<T>
 * (src/composer.cpp:814-976) with Hashing::subgroup_range (src/hashing.h:289-385)
 * restated WITHOUT its remainder-block defect (hashing.h:345) and
 * Partition::histogram_based_reordering (src/partition.h:44-161):
 *   order (in/out): row ids in the previous round's clustered order
 *                   (round 0: order is output only, starts as iota);
 *   in_group:       NULL for round 0, else the previous round's clustered ids;
 *   group_idx:      per position, dense group id numbered by first appearance
 *                   inside each run of equal in_group (intermediate_group_idx);
 *   last_round = 0: order and out_group are re-clustered by group id, stably;
 *   last_round = 1: order is left as is, out_group may be NULL.
 * *ngroups receives the total group count. */
int orc_hash_round(const void *bank, uint32_t bank_bytes, uint32_t *order,
                   const uint32_t *in_group, uint32_t *out_group,
                   uint32_t *group_idx, uint64_t n, int last_round,
                   uint32_t *ngroups);

/* Hash grouping without re-clustering (hash_type 0; Composer::
 * hashByGroup_non_reordered, src/composer.cpp:1153-1219, Hashing::
 * subgroup_first_round / subgroup_non_first_round, src/hashing.h:387-422 and
 * 96-148): out_group[i] = id of (in_group[i], bank[i]) (in_group NULL: bank[i])
 * numbered by first appearance in row order. */
int orc_hash_unordered(const void *bank, uint32_t bank_bytes, const uint32_t *in_group,
                       uint32_t *out_group, uint64_t n, uint32_t *ngroups);

/* Whole plan, sort path: stitch each bank then chain the rounds
 * (run_single_plan, src/stitch_composer.cpp:555-806 + multiRoundSorting,
 * src/composer.cpp:48-135).  cols[c] has col_bytes[c] bytes per row and
 * declared width bw[c]; col_order[k] is the column whose bits come k-th (the
 * reference's columnOrder, src/stitch_composer.cpp:15-35, 568-612; NULL =
 * 0..ncols-1 as in RunAnInstance, src/stitch_composer.cpp:4051-4120).
 * order_out / group_out receive the final order and the final round's group
 * vector (computed even for the last round). */
int orc_run_plan_sort(const void *const *cols, const uint32_t *col_bytes,
                      const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                      const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups);

/* Whole plan, hash path (run_single_plan_hash, src/stitch_composer.cpp:808-1079 +
 * multiRoundHashing_reordered, src/composer.cpp:137-227).  order_out is the
 * last round's input order, group_out the last round's group_idx; col_order as
 * for orc_run_plan_sort. */
int orc_run_plan_hash(const void *const *cols, const uint32_t *col_bytes,
                      const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                      const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups);

#ifdef __cplusplus
}
#endif

#endif /* FMCS_ORACLE_H */
