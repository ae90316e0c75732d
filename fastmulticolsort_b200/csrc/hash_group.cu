// hash_group.cu -- (e) GROUP BY through hashing, one round.
//
// Reference: Composer::hashByGroup_reordered<T> (src/composer.cpp:814-976).
// Per parent group (run of equal in_group) it assigns group ids with a chained
// hash table in order of FIRST APPEARANCE (Hashing::subgroup_range,
// src/hashing.h:289-385; hash mix_int/mix_lng, :21-24), the ids of consecutive
// parent groups continuing from each other (startGrpIdx).  Unless it is the
// last round it then clusters the oids by id with a stable counting scatter
// (Partition::histogram_based_reordering, src/partition.h:44-161).
//
// B200 design.  First-appearance numbering is order-dependent, so it is made
// deterministic without a serial walk:
//   1. one open-addressing table keyed by (parent run, key) over the whole
//      round, one 64-bit word per slot (a fingerprint of the key and the
//      smallest row seen); each row claims or finds its slot and records it,
//      and lowers the slot's row to its own position: the slot's final row is
//      the key's first appearance f(i) inside its run;
//   2. first[i] = (f(i) == i); a one-pass flag scan ranks the first
//      appearances; id(i) = rank(f(i)).  Runs are in position order, so the
//      ranks continue across runs exactly like startGrpIdx;
//   3. the stable clustering is the stable segmented radix sort of
//      (id, oid) inside each run (segsort.cu).
// The hash function only spreads keys over slots; ids never depend on it.
// The reference's remainder-block defect (src/hashing.h:345, every block of a
// range sized `rem_sz`) is not reproduced: every row of every run is grouped.
#include "device_common.cuh"
#include "fmcs_internal.h"

namespace fmcs {

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

template <typename K>
__device__ __forceinline__ K key_at(const K *bank, const uint32_t *order, uint64_t i)
{
    return order ? bank[order[i]] : bank[i];
}

// Table slot: (32-bit fingerprint of (run, key)) << 32 | smallest row seen;
// all ones = empty.  A row claims an empty slot with one CAS (it is then the
// smallest row so far); a row whose fingerprint matches checks the key of the
// slot's row (the only extra read, skipped for keys whose fingerprints differ)
// and lowers the row part with a 64-bit atomicMin (equal fingerprints: only the
// row part can change).  The slot's final row part is the key's first
// appearance inside its run.
constexpr unsigned long long kEmptySlot = ~0ull;
constexpr uint64_t kHashMinSlots = 1024;
constexpr uint64_t kHashMaxSlots = kHashMaxRows;   // slot indices stay below slot_of's sentinels

// slot_of of a row alone in its parent run: it is its own first appearance
// and takes no slot.
constexpr uint32_t kAlone = 0xFFFFFFFFu;

template <typename K>
__global__ void __launch_bounds__(256)
hash_insert_kernel(const K *__restrict__ bank, const uint32_t *__restrict__ order, const uint32_t *__restrict__ run,
                   bool runs_contiguous, const uint32_t *__restrict__ seg_start, uint32_t onchip_max, uint64_t n,
                   unsigned long long *slots, const unsigned long long *d_mask, uint32_t *slot_of, int *status)
{
    kernel_prologue();
    const uint64_t mask = *d_mask;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = run ? run[i] : 0u;
        if (seg_start && seg_start[r + 1] - seg_start[r] <= onchip_max) continue;   // numbered on chip
        if (runs_contiguous && (i == 0 || run[i - 1] != r) && (i + 1 == n || run[i + 1] != r)) {
            slot_of[i] = kAlone;
            continue;
        }
        const K k = key_at(bank, order, i);
        const uint64_t mixed = mix64((uint64_t)k ^ ((uint64_t)r * 0x9E3779B97F4A7C15ull));
        uint64_t h = mixed & mask;
        const uint32_t fp = (uint32_t)(mixed >> 32);
        const unsigned long long mine = ((unsigned long long)fp << 32) | (uint32_t)i;   // never kEmptySlot: i < 2^32 - 1
        uint64_t probes = 0;
        for (;;) {
            unsigned long long cur = *(volatile unsigned long long *)&slots[h];
            if (cur == kEmptySlot) {
                const unsigned long long prev = atomicCAS(&slots[h], kEmptySlot, mine);
                if (prev == kEmptySlot) {
                    slot_of[i] = (uint32_t)h;
                    break;
                }
                cur = prev;
            }
            if ((uint32_t)(cur >> 32) == fp) {
                const uint32_t rr = (uint32_t)cur;   // a row of this slot's (run, key)
                if (key_at(bank, order, rr) == k && (run ? run[rr] : 0u) == r) {
                    // the slot's row only decreases: a smaller row there already wins
                    if (rr > (uint32_t)i) atomicMin(&slots[h], mine);
                    slot_of[i] = (uint32_t)h;
                    break;
                }
            }
            h = (h + 1) & mask;
            if (++probes > mask) {   // table full: cannot happen with more slots than rows
                atomicCAS(status, kDevOk, kDevBadInput);
                slot_of[i] = 0;
                break;
            }
        }
    }
}

// The table's slots set empty: cap_max slots without parent runs, else just
// enough for the rows of the runs the global table takes (counts[2], set by
// the classification; none when every run is numbered on chip).  The mask
// the insert uses is written to *d_mask.
__global__ void hash_table_clear_kernel(unsigned long long *slots, uint64_t cap_max, const uint32_t *counts,
                                        unsigned long long *d_mask)
{
    kernel_prologue();
    uint64_t cap = cap_max;
    if (counts) {
        const uint64_t rows = counts[2];
        cap = rows ? kHashMinSlots : 0;
        while (cap && cap < 2 * rows) cap <<= 1;
        cap = min(cap, cap_max);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_mask = cap ? cap - 1 : 0;
    uint4 *w = reinterpret_cast<uint4 *>(slots);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap / 2; i += stride)
        w[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
}

// slot_of of a row whose parent run was numbered in shared memory: its fpos
// and first flag are written already.
constexpr uint32_t kDoneOnChip = 0xFFFFFFFEu;

// Parent runs of up to kRunOnChip rows are numbered on chip (the reference's
// block-local tables, Hashing::calculate_hash_in_block, src/hashing.h:178-287),
// longer runs in the global table.  A classification pass (one thread per run)
// settles one-row runs at once and queues the others by size: runs of up to
// 32 rows are numbered by one warp each (match.any on the key: a lane's first
// appearance is the lowest lane holding its key), runs of 33 to kRunOnChip rows
// by one CTA each: the run's keys are staged in shared memory, every row claims
// or finds its key's slot of an open-addressing table of positions (at least
// twice as many slots as rows) and lowers the slot to its own position with a
// shared atomicMin, so a slot ends at its key's first appearance in the run.
constexpr uint32_t kRunOnChip = 2048;
constexpr uint32_t kRunOnChipSlots = 2 * kRunOnChip;
constexpr uint32_t kRunWarp = 32;

__global__ void hash_runs_classify_kernel(const uint32_t *__restrict__ seg_start, const uint32_t *d_nseg,
                                          uint32_t *slot_of, uint32_t *fpos, uint8_t *first, uint32_t *warp_runs,
                                          uint32_t *cta_runs, uint32_t *counts)
{
    kernel_prologue();
    const uint32_t nseg = *d_nseg;
    const uint32_t stride = gridDim.x * blockDim.x;
    // every lane of a warp takes the same number of steps (the queue appends
    // below are warp-wide)
    const uint32_t steps = (nseg + stride - 1) / stride;
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t k = 0; k < steps; ++k, s += stride) {
        uint32_t start = 0, len = 0;
        if (s < nseg) {
            start = seg_start[s];
            len = seg_start[s + 1] - start;
        }
        if (len == 1) {
            fpos[start] = start;
            first[start] = 1;
            slot_of[start] = kDoneOnChip;
        }
        const int which = (len >= 2 && len <= kRunWarp) ? 0 : (len > kRunWarp && len <= kRunOnChip) ? 1 : 2;
        const uint32_t lane = threadIdx.x & 31;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, which);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (which < 2 && lane == leader) base = atomicAdd(&counts[which], (uint32_t)__popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        const uint32_t slot = base + __popc(peers & lanemask_lt());
        if (which == 0) warp_runs[slot] = s;
        else if (which == 1) cta_runs[slot] = s;
        // rows of the runs left to the global table (sizes its clear)
        const uint32_t big = __reduce_add_sync(0xFFFFFFFFu, len > kRunOnChip ? len : 0u);
        if (lane == 0 && big) atomicAdd(&counts[2], big);
    }
}

template <typename K>
__global__ void __launch_bounds__(256) hash_runs_onchip_kernel(const K *__restrict__ bank,
                                                               const uint32_t *__restrict__ order,
                                                               const uint32_t *__restrict__ seg_start,
                                                               const uint32_t *warp_runs, const uint32_t *cta_runs,
                                                               const uint32_t *counts, uint32_t *slot_of,
                                                               uint32_t *fpos, uint8_t *first)
{
    kernel_prologue();
    __shared__ K keys[kRunOnChip];
    __shared__ uint32_t table[kRunOnChipSlots];
    __shared__ uint16_t slot_at[kRunOnChip];
    // runs of 33..kRunOnChip rows: one CTA each
    const uint32_t ncta = counts[1];
    for (uint32_t q = blockIdx.x; q < ncta; q += gridDim.x) {
        const uint32_t sidx = cta_runs[q];
        const uint32_t start = seg_start[sidx];
        const uint32_t len = seg_start[sidx + 1] - start;
        uint32_t ts = 64;
        while (ts < 2 * len) ts <<= 1;
        for (uint32_t i = threadIdx.x; i < ts; i += blockDim.x) table[i] = 0xFFFFFFFFu;
        for (uint32_t p = threadIdx.x; p < len; p += blockDim.x)
            keys[p] = order ? bank[order[start + p]] : bank[start + p];
        __syncthreads();
        for (uint32_t p = threadIdx.x; p < len; p += blockDim.x) {
            const K k = keys[p];
            uint32_t h = (uint32_t)mix64((uint64_t)k) & (ts - 1);
            for (uint32_t probe = 0; probe < ts; ++probe) {   // ts > len: a free or matching slot exists
                uint32_t cur = table[h];
                if (cur == 0xFFFFFFFFu) {
                    const uint32_t prev = atomicCAS(&table[h], 0xFFFFFFFFu, p);
                    if (prev == 0xFFFFFFFFu) break;
                    cur = prev;
                }
                if (keys[cur] == k) {
                    atomicMin(&table[h], p);
                    break;
                }
                h = (h + 1) & (ts - 1);
            }
            slot_at[p] = (uint16_t)h;
        }
        __syncthreads();
        for (uint32_t p = threadIdx.x; p < len; p += blockDim.x) {
            const uint32_t f = table[slot_at[p]];
            fpos[start + p] = start + f;
            first[start + p] = f == p ? 1 : 0;
            slot_of[start + p] = kDoneOnChip;
        }
        __syncthreads();
    }
    // runs of 2..32 rows: one warp each, lane i holding row i
    const uint32_t nwarp = counts[0];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x / 32;
    for (uint32_t q = blockIdx.x * wpb + (threadIdx.x >> 5); q < nwarp; q += gridDim.x * wpb) {
        const uint32_t sidx = warp_runs[q];
        const uint32_t start = seg_start[sidx];
        const uint32_t len = seg_start[sidx + 1] - start;
        const bool mine = lane < len;
        const uint32_t valid = __ballot_sync(0xFFFFFFFFu, mine);
        if (mine) {
            const K k = order ? bank[order[start + lane]] : bank[start + lane];
            const uint32_t peers = __match_any_sync(valid, (unsigned long long)k);
            const uint32_t f = __ffs(peers) - 1;
            fpos[start + lane] = start + f;
            first[start + lane] = f == lane ? 1 : 0;
            slot_of[start + lane] = kDoneOnChip;
        }
    }
}

__global__ void first_flag_kernel(const uint32_t *__restrict__ slot_of, const unsigned long long *__restrict__ slots,
                                  uint8_t *__restrict__ first, uint32_t *__restrict__ fpos, uint64_t n)
{
    kernel_prologue();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t so = slot_of[i];
        if (so == kDoneOnChip) continue;
        const uint32_t f = so == kAlone ? (uint32_t)i : (uint32_t)slots[so];
        fpos[i] = f;
        first[i] = (f == (uint32_t)i) ? 1 : 0;
    }
}

// id(i) = rank(f(i)); with `row_ids` also scatter the id to the row it
// belongs to (row-indexed, the layout the segmented sort gathers from).
// With `clustered` (a word that starts non-zero), a position whose id is
// smaller than its predecessor's clears it: the ids of consecutive runs
// ascend, so a word still set at the end says that every run's rows are in
// id order already and the stable clustering moves nothing.  With
// `key_bits`, the bits of the largest id (the group count less one).
__global__ void assign_ids_kernel(const uint32_t *__restrict__ fpos, const uint32_t *__restrict__ rank,
                                  const uint32_t *__restrict__ order, uint32_t *__restrict__ ids,
                                  uint32_t *__restrict__ row_ids, uint64_t n, uint32_t *clustered,
                                  const uint32_t *d_ngroups, uint32_t *key_bits)
{
    kernel_prologue();
    if (key_bits && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t g = *d_ngroups;
        *key_bits = g <= 1 ? 0u : 32u - (uint32_t)__clz(g - 1);
    }
    bool descent = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = rank[fpos[i]];
        if (ids) ids[i] = g;
        if (row_ids) row_ids[order ? order[i] : (uint32_t)i] = g;
        if (clustered && i > 0 && rank[fpos[i - 1]] > g) descent = true;
    }
    if (clustered && __any_sync(0xFFFFFFFFu, descent) && (threadIdx.x & 31) == 0) *clustered = 0u;
}

// The round's numbering: with parent-run starts (seg_start, *d_nseg runs),
// runs of up to kRunOnChip rows in shared memory, the others in the global
// table; without, every row in the global table.  The table (cap_max slots
// allocated) is cleared only as far as the rows it takes need.
template <typename K>
int hash_insert(fmcs_ctx *ctx, const void *bank, const uint32_t *order, const uint32_t *run, bool runs_contiguous,
                const uint32_t *seg_start, const uint32_t *d_nseg, uint64_t n, unsigned long long *slots,
                uint64_t cap_max, unsigned long long *d_mask, uint32_t *slot_of, uint32_t *fpos, uint8_t *first,
                uint32_t *warp_runs, uint32_t *cta_runs, uint32_t *counts)
{
    const unsigned grid = (unsigned)ctx->num_sms * 8;
    if (seg_start) {
        cudaMemsetAsync(counts, 0, 3 * sizeof(uint32_t), ctx->stream);
        {
            LaunchScope ls_(ctx, "hash_runs_classify");
            launch_k(hash_runs_classify_kernel, grid, 256, 0, ctx->stream, seg_start, d_nseg, slot_of, fpos, first,
                     warp_runs, cta_runs, counts);
        }
        LaunchScope ls_(ctx, "hash_runs_onchip");
        launch_k(hash_runs_onchip_kernel<K>, grid, 256, 0, ctx->stream, (const K *)bank, order, seg_start,
                 (const uint32_t *)warp_runs, (const uint32_t *)cta_runs, (const uint32_t *)counts, slot_of, fpos,
                 first);
    }
    { LaunchScope ls_(ctx, "hash_table_clear");
        launch_k(hash_table_clear_kernel, grid, 256, 0, ctx->stream, slots, cap_max,
                 (const uint32_t *)(seg_start ? counts : nullptr), d_mask);
    }
    { LaunchScope ls_(ctx, "hash_insert");
        launch_k(hash_insert_kernel<K>, grid, 256, 0, ctx->stream, (const K *)bank, order, run, runs_contiguous,
                 seg_start, kRunOnChip, n, slots, (const unsigned long long *)d_mask, slot_of, ctx->d_status);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "hash insert launch");
}

}  // namespace

int hash_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, const uint32_t *order_in,
               uint32_t *order_out, const uint32_t *in_group, uint32_t *out_group, uint64_t n, bool last_round,
               uint32_t *d_ngroups, bool group_is_key, bool fixed_launches)
{
    if (n == 0) return FMCS_OK;
    if (n >= kHashMaxSlots) return set_error(ctx, FMCS_E_INVAL, "hash round: at most 2^31 - 1 rows");
    cudaStream_t st = ctx->stream;
    int rc;
    void *p;
    // table: up to cap 64-bit slots (at least twice the rows, at most 2^31;
    // always more slots than rows), cleared on the device by hash_insert
    uint64_t cap = kHashMinSlots;
    while (cap < 2 * n && cap < kHashMaxSlots) cap <<= 1;
    if ((rc = ws_get(ctx, kSlotHashTable, cap * sizeof(unsigned long long), &p))) return rc;
    unsigned long long *slots = (unsigned long long *)p;
    // per-row scratch: slot_of / rank, fpos, run ids, first flags; and the
    // queues of parent runs numbered on chip (a warp each: at most n / 2 runs
    // of 2..32 rows; a CTA each: at most n / 33)
    const uint64_t nq_warp = n / 2 + 1, nq_cta = n / (kRunWarp + 1) + 1;
    if ((rc = ws_get(ctx, kSlotHashIdx,
                     carve_total({n * sizeof(uint32_t), n * sizeof(uint32_t), n * sizeof(uint32_t), n,
                                  nq_warp * sizeof(uint32_t), nq_cta * sizeof(uint32_t)}),
                     &p)))
        return rc;
    Carver cv(p);
    uint32_t *slot_of = cv.take<uint32_t>(n);
    uint32_t *fpos = cv.take<uint32_t>(n);
    uint32_t *run = cv.take<uint32_t>(n);
    uint8_t *first = cv.take<uint8_t>(n);
    uint32_t *warp_runs = cv.take<uint32_t>(nq_warp);
    uint32_t *cta_runs = cv.take<uint32_t>(nq_cta);
    if ((rc = ws_get(ctx, kSlotCounters, 4096, &p))) return rc;
    uint32_t *d_cnt = (uint32_t *)p + 32;   // words 32..39 and 48..49 belong to the hash round
    unsigned long long *d_mask = reinterpret_cast<unsigned long long *>((uint32_t *)p + 48);
    uint32_t *seg_start = nullptr;
    // The key of a row is (its parent run, its value): the run id from a
    // boundary scan of in_group, or -- when the previous ids are not clustered
    // (group_is_key) -- the previous id itself, over one numbering in row order.
    const uint32_t *keyrun = nullptr;
    bool contiguous = false;   // runs are position ranges (not the previous ids of unclustered rows)
    if (in_group && group_is_key) {
        keyrun = in_group;
    } else if (in_group) {
        // run ids and run starts in one boundary scan of in_group
        if ((rc = ws_get(ctx, kSlotSegStart, (n + 2) * sizeof(uint32_t), &p))) return rc;
        seg_start = (uint32_t *)p;
        if ((rc = launch_group_ids_segments(ctx, nullptr, 0, in_group, run, seg_start, n, d_cnt))) return rc;
        keyrun = run;
        contiguous = true;
    }
    switch (bank_bytes) {
    case 1: rc = hash_insert<uint8_t>(ctx, bank, order_in, keyrun, contiguous, seg_start, d_cnt, n, slots, cap,
                                      d_mask, slot_of, fpos, first, warp_runs, cta_runs, d_cnt + 4); break;
    case 2: rc = hash_insert<uint16_t>(ctx, bank, order_in, keyrun, contiguous, seg_start, d_cnt, n, slots, cap,
                                       d_mask, slot_of, fpos, first, warp_runs, cta_runs, d_cnt + 4); break;
    case 4: rc = hash_insert<uint32_t>(ctx, bank, order_in, keyrun, contiguous, seg_start, d_cnt, n, slots, cap,
                                       d_mask, slot_of, fpos, first, warp_runs, cta_runs, d_cnt + 4); break;
    case 8: rc = hash_insert<uint64_t>(ctx, bank, order_in, keyrun, contiguous, seg_start, d_cnt, n, slots, cap,
                                       d_mask, slot_of, fpos, first, warp_runs, cta_runs, d_cnt + 4); break;
    default: return set_error(ctx, FMCS_E_INVAL, "hash round: bank_bytes must be 1, 2, 4 or 8");
    }
    if (rc) return rc;
    const unsigned grid = (unsigned)ctx->num_sms * 8;
    { LaunchScope ls_(ctx, "first_flag");
        launch_k(first_flag_kernel, grid, 256, 0, st, slot_of, slots, first, fpos, n);
    }
    uint32_t *rank = slot_of;   // slot_of is dead after the flags
    if ((rc = launch_flag_rank(ctx, first, rank, n, d_ngroups))) return rc;
    if (last_round) {
        { LaunchScope ls_(ctx, "assign_ids");
            launch_k(assign_ids_kernel, grid, 256, 0, st, fpos, rank, nullptr, out_group, nullptr, n, nullptr,
                     (const uint32_t *)d_ngroups, nullptr);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(ctx, e, "hash ids launch");
        if (order_out != order_in) {
            if (order_in)
                cudaMemcpyAsync(order_out, order_in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
            else
                return set_error(ctx, FMCS_E_INVAL, "hash round: internal order");
        }
        return FMCS_OK;
    }
    // clustering: stable sort of (id, oid) inside each parent run; ids are
    // scattered to row order so that the sort's gather through order_in reads them.
    uint32_t *row_ids = run;   // run ids are dead after the insert
    // the sort's key width (the bits of the largest id) and whether the ids
    // are in order already are decided on the device: no read-back
    uint32_t *d_clustered = d_cnt + 2, *d_kbits = d_cnt + 3;
    cudaMemsetAsync(d_clustered, 0xFF, sizeof(uint32_t), st);
    { LaunchScope ls_(ctx, "assign_ids");
        launch_k(assign_ids_kernel, grid, 256, 0, st, fpos, rank, order_in, nullptr, row_ids, n, d_clustered,
                 (const uint32_t *)d_ngroups, d_kbits);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "hash ids launch");
    uint32_t bits = 1;   // ids < n: a bound on the key width, which sets the most radix levels
    while (bits < 32 && (1ull << bits) < n) bits++;
    if (in_group && !seg_start) {
        // previous ids as the key (unclustered rows): the clustering's segments
        // are still the runs of equal in_group
        if ((rc = ws_get(ctx, kSlotSegStart, (n + 2) * sizeof(uint32_t), &p))) return rc;
        seg_start = (uint32_t *)p;
        if ((rc = launch_segments(ctx, in_group, seg_start, d_cnt, n))) return rc;
    }
    SortArgs a;
    a.bank = row_ids;
    a.bank_bytes = 4;
    a.key_bits = bits;
    a.order_in = order_in;
    a.seg_start = seg_start;
    a.nseg_host = 0;
    a.d_nseg = seg_start ? d_cnt : nullptr;
    a.order_out = order_out;
    a.keys_out = out_group;
    a.n = n;
    a.fixed_launches = fixed_launches;
    a.d_key_bits = d_kbits;
    a.d_in_order = d_clustered;
    return sort_segments(ctx, a);
}

}  // namespace fmcs
