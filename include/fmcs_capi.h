/*
 * fmcs_capi.h -- C ABI of the B200 multi-column sort path.
 *
 * The reference (FastMultiColSort) has no FFI: it is a static C++ library whose
 * swap points are the Composer virtuals SortAllColumns_Nonpack / HashAllColumns
 * (src/composer.h:59-68) and StitchComposer::run_single_plan, which hard-codes a
 * CPU ChainComposer (src/stitch_composer.cpp:745, 1009).  Each entry point below
 * names the reference code it replaces.  The C++ classes in include/fmcs/ that
 * mirror the reference's Column / ChainComposer / StitchComposer API sit on top
 * of this ABI.
 *
 * Conventions
 *   - Row ids (oids), order and group vectors are uint32 (surrogate_t,
 *     src/params.h:9-13); n < 2^32.  Hash rounds (and hash plans) take
 *     n < 2^31: their table holds up to 2^31 slots with 32-bit indices.
 *   - Banks are 1, 2, 4 or 8 bytes per row (sort rounds: 2, 4 or 8).
 *   - Pointers may be device pointers or host pointers (pageable or pinned);
 *     host data is staged through the context's device buffers, so a host
 *     call pays its own copies.  Inputs are never modified.
 *   - All calls are stream-ordered on the context's stream and return after the
 *     results are complete (host outputs) or enqueued (device outputs; call
 *     fmcs_synchronize before reading them from another stream).
 *   - Status codes: FMCS_OK 0, FMCS_E_INVAL -1, FMCS_E_OOM -2,
 *     FMCS_E_TIMEOUT -3 (a bounded device-side wait gave up), FMCS_E_CUDA -4.
 *     fmcs_last_error() gives the message of the last failure.
 *   - A context is not thread-safe; use one per host thread.
 */
#ifndef FMCS_CAPI_H
#define FMCS_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FMCS_API __attribute__((visibility("default")))
#else
#define FMCS_API
#endif

#define FMCS_OK 0
#define FMCS_E_INVAL (-1)
#define FMCS_E_OOM (-2)
#define FMCS_E_TIMEOUT (-3)
#define FMCS_E_CUDA (-4)

typedef struct fmcs_ctx fmcs_ctx;

/* Create a context on `device`.  hbm_budget_bytes caps the context's device
 * workspace (0 = no cap).  Replaces the reference's per-call malloc_aligned
 * (src/common.h:18-31). */
FMCS_API int fmcs_create(fmcs_ctx **ctx, int device, size_t hbm_budget_bytes);
FMCS_API void fmcs_destroy(fmcs_ctx *ctx);
FMCS_API const char *fmcs_last_error(const fmcs_ctx *ctx);
/* Wait for all work of the context (its stream). */
FMCS_API int fmcs_synchronize(fmcs_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work against it. */
FMCS_API void *fmcs_stream(fmcs_ctx *ctx);
/* Device bytes the context currently holds in its workspace. */
FMCS_API size_t fmcs_workspace_bytes(const fmcs_ctx *ctx);

/* Kernel profiler (no reference counterpart; the reference times sections with
 * rdtsc, src/hybrid_timer.h:16-56).  While enabled, every kernel launch of the
 * context is bracketed by CUDA events on its stream.  fmcs_profile_report
 * synchronizes and writes a JSON object
 * {"kernel": {"launches": n, "ms": t, "units": u}} for the launches since the
 * last report, then forgets them; units are the rows the launches processed
 * where the launcher knows them (the MSD scatter passes), else 0. */
FMCS_API int fmcs_profile(fmcs_ctx *ctx, int enable);
FMCS_API int fmcs_profile_report(fmcs_ctx *ctx, char *buf, size_t len);
/* Self-test of the bounded device waits (no reference counterpart; the
 * reference has no device code).  Every device-side wait of the library (the
 * decoupled look-backs) polls a bounded number of times, then records
 * FMCS_E_TIMEOUT in the context's status word and lets its kernel finish.
 * This call runs that same wait on a word that nothing writes, with a limit of
 * `polls` polls (1..2^20), and returns what the host then reads:
 * FMCS_E_TIMEOUT, with the status word cleared and the context usable. */
FMCS_API int fmcs_selftest_wait(fmcs_ctx *ctx, uint32_t polls);
/* Number of kernels this context has launched since it was created. */
FMCS_API unsigned long long fmcs_launch_count(const fmcs_ctx *ctx);

/* Tuned knobs of the sort engine (no reference counterpart; the reference's
 * block sizes are compile-time constants, src/params.h:127-143).  A context
 * starts from the autotuner's file (tuning/b200.json next to the library, or
 * the file FMCS_TUNING names), else the built-in defaults.  Keys:
 *   "rank_mode"  0: match.any multi-split ranking, 1: ballot multi-split,
 *                2: shared-memory OR peer words (HBM radix levels; ballot elsewhere);
 *   "local_max"  128..8192: segments with more rows take the HBM radix levels;
 *   "msd_items"  8 or 16: items per thread of an HBM radix tile.
 * fmcs_get_tuning returns -1 for an unknown key. */
FMCS_API int fmcs_set_tuning(fmcs_ctx *ctx, const char *key, long long value);
FMCS_API long long fmcs_get_tuning(const fmcs_ctx *ctx, const char *key);

/* One slice of a source column: bits [start, end], 1-based from the MSB of the
 * declared width src_bits (construct_entry_t, src/types.h:42-46). */
typedef struct {
    const void *src;
    uint32_t src_bytes; /* 1, 2, 4 or 8 */
    uint32_t src_bits;  /* declared width of the source column, <= 8*src_bytes */
    uint32_t start;
    uint32_t end;
} fmcs_slice;

/* (a) Bit stitching of one bank: ShiftLeftBatch + AssembleFromColumn for every
 * slice (src/column.h:105-180, 208-1060; loop at src/stitch_composer.cpp:655-703).
 * bank: n rows of bank_bytes. */
FMCS_API int fmcs_stitch(fmcs_ctx *ctx, const fmcs_slice *slices, uint32_t nslices,
                void *bank, uint32_t bank_bytes, uint64_t n);

/* Slice-at-a-time bank building, exactly the reference's two whole-column
 * primitives (for code that builds banks itself; fmcs_stitch is the fused
 * one-pass form):
 *   fmcs_shift_left: bank[i] <<= nbits, truncated to the bank width
 *                    (SpecialiedColumn<T>::ShiftLeftBatch, src/column.h:105-180);
 *   fmcs_assemble:   bank[i] |= (src[i] >> (src_bits - end)) & mask(end-start+1)
 *                    (SpecialiedColumn<T>::AssembleFromColumn, src/column.h:208-1060). */
FMCS_API int fmcs_shift_left(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n, uint32_t nbits);
FMCS_API int fmcs_assemble(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n,
                           const fmcs_slice *slice);

/* (c) out[i] = bank[order[i]] (Composer::BATproject, src/composer.cpp:608-628). */
FMCS_API int fmcs_gather(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes,
                const uint32_t *order, void *out, uint64_t n);

/* (b)+(d) One sort round (Composer::sortByGroup<T>, src/composer.cpp:1222-1408,
 * with subsort (:558-589) and extractGroupInfo (:630-678)).
 *   in_group == NULL: round 0; order is output only (the reference starts
 *                     from iota, :60-63) and receives the stable argsort of bank.
 *   in_group != NULL: order is input and output; the round sorts bank[order[i]]
 *                     stably inside every run of equal in_group.
 *   key_bits:         significant bits of the bank (1..8*bank_bytes); bits above
 *                     must be zero.
 *   out_group:        dense group ids in sorted order, or NULL for a last round
 *                     (isLastRound, :1388-1390).
 *   sorted_bank:      optional (NULL): receives the sorted bank values.
 *   ngroups:          optional: receives the group count (0 if out_group NULL).
 * Ties keep their input order, which equals the reference's result with ties
 * canonicalised to ascending oid. */
FMCS_API int fmcs_sort_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t key_bits,
                    uint32_t *order, const uint32_t *in_group, uint32_t *out_group,
                    void *sorted_bank, uint64_t n, uint32_t *ngroups);

/* The plain comparator of one sort round: same inputs, outputs and results
 * as fmcs_sort_round, computed WITHOUT segments -- a full-array stable LSD
 * radix sort by the key, then (later rounds) a full-array stable LSD radix
 * sort by the previous group id.  This is the "one sort per column" GPU path
 * that the segmented, size-binned rounds are measured against; it has no
 * reference counterpart (the reference always sorts per group,
 * src/composer.cpp:1280-1335). */
FMCS_API int fmcs_sort_round_plain(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t key_bits,
                                   uint32_t *order, const uint32_t *in_group, uint32_t *out_group,
                                   void *sorted_bank, uint64_t n, uint32_t *ngroups);

/* (e) One hash-grouping round (Composer::hashByGroup_reordered<T>,
 * src/composer.cpp:814-976; Hashing::subgroup_range, src/hashing.h:289-385;
 * Partition::histogram_based_reordering, src/partition.h:44-161).
 *   in_group == NULL: round 0, order output only (starts as iota).
 *   group ids are dense, numbered by first appearance inside each run of equal
 *   in_group, runs in position order (startGrpIdx accumulates).
 *   last_round == 0:  order and out_group are re-clustered by group id, stably.
 *   last_round != 0:  order is left as is; out_group gets the per-position group
 *                     ids (intermediate_group_idx).
 * The reference's remainder-block defect (src/hashing.h:345) is not reproduced. */
FMCS_API int fmcs_hash_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes,
                    uint32_t *order, const uint32_t *in_group, uint32_t *out_group,
                    uint64_t n, int last_round, uint32_t *ngroups);

/* (e) One hash-grouping round WITHOUT re-clustering (hash_type 0:
 * Composer::hashByGroup_non_reordered, src/composer.cpp:1153-1219, with
 * Hashing::subgroup_first_round / subgroup_non_first_round, src/hashing.h:387-422,
 * 96-148): out_group[i] = dense id of the pair (in_group[i], bank[i]) numbered
 * by first appearance in ROW order (in_group NULL: of bank[i] alone). */
FMCS_API int fmcs_hash_round_unordered(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes,
                                       const uint32_t *in_group, uint32_t *out_group, uint64_t n,
                                       uint32_t *ngroups);

/* Whole massaged plan (StitchComposer::run_single_plan,
 * src/stitch_composer.cpp:555-806 + multiRoundSorting, src/composer.cpp:48-135,
 * or with hash != 0 run_single_plan_hash, :808-1079 + multiRoundHashing_reordered,
 * src/composer.cpp:137-227).
 *   cols[c]:    n rows of col_bytes[c] bytes, declared width bw[c];
 *               col_order (NULL = 0..ncols-1) is the reference's columnOrder.
 *   split:      bank widths in bits (sum == sum of bw), e.g. {50} or {6,44}.
 *   order_out:  final order; group_out: group vector of the last round
 *               (always computed; NULL to skip).  ngroups optional. */
FMCS_API int fmcs_run_plan(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes,
                  const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                  const uint32_t *split, uint32_t nbanks, uint64_t n, int hash,
                  uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups);

/* fmcs_run_plan with a sort direction per column: descending[c] != 0 sorts
 * column c in descending order (NULL: all ascending).  The reference parses a
 * per-column direction (compose_params_t::column_asc_desc, --asc-desc in
 * src/main_tworound_exhaustive.cpp:347-376) but sorts every column
 * ascending; here the stitch inverts the column's bits inside its declared
 * width, so a descending column orders by (2^bw - 1 - value) and ties still
 * keep their input order.  With hash != 0 the groups are the same as with
 * every column ascending. */
FMCS_API int fmcs_run_plan_desc(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes,
                                const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                                const uint8_t *descending, const uint32_t *split, uint32_t nbanks, uint64_t n,
                                int hash, uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups);

/* Per-group aggregates of a payload column: the consumer of (order, group)
 * that GROUP BY queries run next (the reference returns (order, group) only,
 * Composer::getGroupInfo, src/composer.h:59-68).  For every sorted position i
 * the payload value of row order[i] joins group group[i] (< ngroups); outputs
 * of ngroups entries each, any may be NULL: count, sum (64-bit, wrapping; the
 * signed sum for signed payloads when it does not overflow), min and max
 * (sign-extended when is_signed).  payload: n values of 4 or 8 bytes in row
 * order.  All arrays device memory.  Groups need not be runs of positions (a
 * hash plan's last round is accepted too).  A group id >= ngroups or an order
 * entry >= n is reported as FMCS_E_INVAL, with nothing read or written there. */
FMCS_API int fmcs_group_aggregate(fmcs_ctx *ctx, const void *payload, uint32_t payload_bytes, int is_signed,
                                  const uint32_t *order, const uint32_t *group, uint64_t n, uint32_t ngroups,
                                  uint64_t *count, uint64_t *sum, uint64_t *min, uint64_t *max);

/* The reference's text datasets, on the host (DataGenerator::ReadFromFile,
 * ReadFromFile_tpch, ReadValues and GenAndSaveAsFile, src/generator.h:43-227):
 * unsigned decimal values separated by white space, all rows of column 0,
 * then of column 1, ...; the TPC-H variant starts with the row count and the
 * column count.  Columns are stored in the width their bit width maps to
 * (src/generator.h:88-94): fmcs_storage_bytes(bw) = 2 (bw <= 16), 4 (<= 32)
 * or 8.  No GPU is involved.  Return FMCS_E_INVAL for a missing file,
 * malformed text, a value too large for its column's storage, or a TPC-H
 * header whose row count differs from nrows. */
FMCS_API uint32_t fmcs_storage_bytes(uint32_t bw);
/* Row and column counts of a TPC-H-variant file. */
FMCS_API int fmcs_text_header(const char *path, uint64_t *nrows, uint32_t *ncols);
/* Reads nrows values of each of ncols columns into caller-allocated host
 * arrays cols_out[c] (fmcs_storage_bytes(bw[c]) bytes per value); with
 * cardinality_out, also each column's number of distinct values (the
 * reference's Column::GetCardinality). */
FMCS_API int fmcs_read_columns_text(const char *path, int has_header, uint32_t ncols, const uint32_t *bw,
                                    uint64_t nrows, void *const *cols_out, uint64_t *cardinality_out);
/* Writes columns (host, 2/4/8 bytes per value) in the same format, one value
 * per line, with the TPC-H header when with_header. */
FMCS_API int fmcs_write_columns_text(const char *path, int with_header, uint32_t ncols, uint64_t nrows,
                                     const void *const *cols, const uint32_t *col_bytes);

/* A whole sort plan captured once as a CUDA graph and replayed (no reference
 * counterpart).  The graph is bound to the DEVICE buffers given here (columns,
 * order_out, group_out): refill the columns between launches and replay.
 * It runs in a private context (own stream and workspace, sized by one eager
 * run at creation); every radix level is part of the graph and exits on the
 * device when it has no work, so a replay needs no host round trip until its
 * final status check.  fmcs_graph_create_hash captures the same plan
 * through the hash-grouping rounds (run_single_plan_hash,
 * src/stitch_composer.cpp:808-1079), whose key widths and clustering are also
 * decided on the device.  fmcs_graph_launch returns when the results are
 * complete; fmcs_graph_stream is the graph's stream. */
typedef struct fmcs_graph fmcs_graph;
FMCS_API int fmcs_graph_create(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes,
                               const uint32_t *bw, uint32_t ncols, const uint32_t *col_order, const uint32_t *split,
                               uint32_t nbanks, uint64_t n, uint32_t *order_out, uint32_t *group_out,
                               fmcs_graph **graph);
FMCS_API int fmcs_graph_create_hash(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes,
                                    const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                                    const uint32_t *split, uint32_t nbanks, uint64_t n, uint32_t *order_out,
                                    uint32_t *group_out, fmcs_graph **graph);
FMCS_API int fmcs_graph_launch(fmcs_graph *graph, uint32_t *ngroups);
FMCS_API void *fmcs_graph_stream(fmcs_graph *graph);
/* Kernel nodes of the graph, each loop body (the radix levels of a sort round,
 * a conditional WHILE node that runs as many times as the data needs) counted once. */
FMCS_API int fmcs_graph_kernels(fmcs_graph *graph);
FMCS_API void fmcs_graph_destroy(fmcs_graph *graph);

/* Many independent sort instances in one batch (no reference counterpart: the
 * reference sorts one relation per process).  Instance k holds rows
 * [inst[k].row_off, inst[k].row_off + inst[k].n) of the shared column arrays;
 * instances are contiguous and in row order and share the plan (bw, split).
 * Every instance is one segment of the same size-binned launches.  Outputs
 * are per-instance ranges of order_out / group_out at the same row offsets,
 * with oids and group ids LOCAL to the instance; ngroups_out[k] (optional,
 * host) gets instance k's group count. */
typedef struct {
    uint64_t row_off;
    uint64_t n;
} fmcs_instance;

FMCS_API int fmcs_run_batch(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                            uint32_t ncols, const uint32_t *split, uint32_t nbanks, const fmcs_instance *inst,
                            uint32_t ninst, uint64_t total_rows, uint32_t *order_out, uint32_t *group_out,
                            uint32_t *ngroups_out);

/* The cost-model plan search alone (StitchComposer::optimizeAndRun without
 * the run, src/stitch_composer.cpp:3839-3984): given each column's declared
 * width, number of distinct values and storage bytes, returns the estimated
 * cheapest split (split_out, *nbanks_out <= max_banks) and, for GROUP BY
 * (ordered == 0, columns may be permuted), the column order.  Costs come from
 * the GPU tables (tuning/b200.json next to the library, or FMCS_TUNING).
 * The model assumes the values of a column split the rows into equal groups;
 * for a skewed column pass its effective cardinality n^2 / sum(count^2) over
 * its values' row counts (the number of equal groups with the same mean group
 * size per row) instead of its distinct count: a Zipf(1.0) column of 2^20
 * codes in 67M rows has about 1M distinct values but an effective cardinality
 * near 127, and only the latter predicts how far its groups split. */
FMCS_API int fmcs_optimize_plan(const uint32_t *bw, const uint64_t *cardinality, const uint32_t *col_bytes,
                                uint32_t ncols, uint64_t n, int ordered, uint32_t *split_out, uint32_t max_banks,
                                uint32_t *nbanks_out, uint32_t *col_order_out, double *est_ms);

/* The cost model's estimate (ms on this GPU) of one given plan: split[0..nbanks)
 * over the columns in col_order (NULL = as given), the same tables and the
 * same per-round model as fmcs_optimize_plan's search (StitchComposer::
 * EstimatePlan; the reference estimates plans in StitchComposer::
 * cost_estimation, src/stitch_composer.cpp:2929-3166).  The split must cover
 * the columns' bits exactly. */
FMCS_API int fmcs_estimate_plan(const uint32_t *bw, const uint64_t *cardinality, const uint32_t *col_bytes,
                                uint32_t ncols, uint64_t n, const uint32_t *col_order, const uint32_t *split,
                                uint32_t nbanks, double *est_ms);

/* Allocation-free group ids (no counterpart in the reference, which mallocs
 * on every call).  For callers that cannot let a library allocate device
 * memory: engines that reserve all of HBM in their own pool up front, and
 * latency-critical callers that cannot take the device-wide synchronization of
 * cudaMalloc/cudaFree.  Computes the same dense group ids as the group vector
 * of fmcs_sort_round, from keys that are already sorted inside each run of
 * equal in_group (in_group may be NULL):
 *   out_group[0] = 0; out_group[i] = out_group[i-1] +
 *       (keys[i] != keys[i-1] || in_group[i] != in_group[i-1]).
 * keys, in_group and out_group must be DEVICE pointers of the current device
 * (host pointers are rejected, as staging them would allocate, and so is
 * another GPU's memory); stream is a cudaStream_t (NULL = the default stream);
 * *ngroups (optional, host) receives the group count.  The call is
 * synchronous: it waits for the stream and returns when the result is
 * complete.
 * Scratch lives in a file-scope device array of the library (128 KiB, held by
 * every GPU that loads the library until exit), so n is limited to
 * 67,108,864 rows; larger n returns FMCS_E_INVAL.  The first call on a device
 * resolves that array's device address (cudaGetSymbolAddress), so make that
 * first call on each device before any stream capture begins there.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialized by the caller.  Nothing is allocated: no cudaMalloc, no cudaFree,
 * no allocating library routine. */
FMCS_API int fmcs_group_ids_noalloc(void *stream, const void *keys, uint32_t key_bytes,
                                    const uint32_t *in_group, uint32_t *out_group, uint64_t n,
                                    uint32_t *ngroups);

#ifdef __cplusplus
}
#endif

#endif /* FMCS_CAPI_H */
