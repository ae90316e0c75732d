// segsort.cu -- (b) the per-round sort: a stable, segmented radix sort of
// (bank key, oid) pairs in HBM.
//
// Reference: Composer::sortByGroup<T> (src/composer.cpp:1222-1408) walks the
// previous round's groups and calls subsort -> Mergesort::avxmergesort_anytype
// (src/mergesort.h:2878-3096) once per group: block sorts with AVX2 bitonic
// networks, then 2-way merges, mallocing four buffers per group.  Round 0 is
// one group of n rows.
//
// B200 design.  Every group is a segment [start, start+len) that is sorted in
// place (segments never move).  Segments are binned by size:
//   tier A  len <= 128   one warp per segment, LSD radix in registers/smem
//   tier B  len <= 1024  one 128-thread CTA per segment, LSD radix in smem
//   tier C  len <= 4096  one 256-thread CTA per segment, LSD radix in smem
//   large   len >  4096  MSD radix levels: per-segment digit histogram, then a
//                        onesweep-style stable scatter with a decoupled
//                        look-back chained over the segment's tiles; every
//                        non-empty bucket becomes a child segment with 8 bits
//                        fewer, re-binned into the tiers above.
// Each key is ranked by warp-level multi-split (match.any + popc) so every
// pass is stable; the MSD scatter is stable too, so the whole sort is stable:
// ties keep the oid order of the input, which is what the reference gives once
// its ties are canonicalised to ascending oid.  Rows move only through HBM in
// the large tier; a tier-A/B/C segment is read once and written once.
//
// Data sources of a segment: BUF0 (final buffer: the caller's order array and
// the sorted-key array), BUF1 (work buffer), EXT (the round's input: the bank
// gathered through the previous order, Composer::BATproject at
// src/composer.cpp:608-628, or the bank itself with iota oids in round 0).
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <algorithm>
#include <functional>
#include <vector>

namespace fmcs {

namespace {

constexpr uint32_t kSrcBuf0 = 0;
constexpr uint32_t kSrcBuf1 = 1;
constexpr uint32_t kSrcExt = 2;
constexpr uint32_t kSkipBit = 0x100;

// Local tiers: a segment goes to the smallest tier whose capacity holds it, so
// that each kernel's unrolled item steps match the segment (few idle steps).
constexpr int kCapT = 16;    // thread per segment: registers, odd-even transposition network
constexpr int kCapT32 = 32;  // the same up to 32 rows, for 2- and 4-byte keys (own kernel: more registers)
constexpr int kCapA = 128;   // warp per segment: 32 lanes x 4 items
constexpr int kItemsA = 4;
constexpr int kNtB1 = 128, kItB1 = 4, kCapB1 = kNtB1 * kItB1;   // 512
constexpr int kNtB2 = 128, kItB2 = 8, kCapB2 = kNtB2 * kItB2;   // 1024
constexpr int kNtC1 = 256, kItC1 = 8, kCapC1 = kNtC1 * kItC1;   // 2048
constexpr int kNtC1b = 256, kItC1b = 9, kCapC1b = kNtC1b * kItC1b;   // 2304
constexpr int kNtC2 = 512, kItC2 = 8, kCapC2 = kNtC2 * kItC2;   // 4096
constexpr int kNtC3 = 1024, kItC3 = 8, kCapC3 = kNtC3 * kItC3;  // 8192
constexpr int kCapLocal = kCapC3;   // largest segment a local tier can take; larger: MSD levels
constexpr int kNtM = 256;           // MSD tile: 256 threads x IT items (IT = 8 or 16, tuned)
constexpr int kHistCtas = 4;         // resident histogram CTAs per SM (the grid is one wave)
constexpr int kMsdCtas16 = 3;       // resident scatter CTAs per SM with 16 rows per thread

// counters slot words
constexpr int kCtrMsdTile = 1;
constexpr int kCtrLarge0 = 2;   // + level parity
constexpr int kCtrLocalA = 4;
constexpr int kCtrLocalB1 = 5;
constexpr int kCtrLocalB2 = 6;
constexpr int kCtrCopy = 7;
constexpr int kCtrMoved = 8;    // rows the current level's scatter moves
constexpr int kCtrLocalC1 = 9;
constexpr int kCtrLocalC2 = 10;
constexpr int kCtrLocalT = 11;
constexpr int kCtrLocalT32 = 14;
constexpr int kCtrCopyLarge = 12;   // copy entries larger than kCopySplit rows
constexpr int kCtrCopyTile = 13;
constexpr uint32_t kCopySplit = 4096;
constexpr int kCtrLevel = 15;      // MSD levels started so far (device-side level index)
constexpr int kCtrLocalC3 = 16;
constexpr int kCtrLocalC1b = 17;
constexpr int kCtrChunks0 = 18;    // + level parity: histogram rows (chunks) of the level's large segments
constexpr int kCtrWords = 32;

// An HBM level cuts each large segment's look-back chain every kChunkTiles
// tiles.  Each chunk has its own histogram row; msd_plan turns the rows of a
// segment into per-chunk digit bases (the segment's offset of the digit plus
// the digit's rows in the segment's earlier chunks), so a chunk's first tile
// publishes its inclusive prefix at once and no tile walks back past its
// chunk's start.  One long chain (a round's single segment of thousands of
// tiles) makes every tile wait on the whole GPU's progress; short chains run
// side by side (one level over 16.8M rows: 0.164 ms as one segment, 0.137 ms
// as 256 segments of 16 tiles).  Chunks of 32 tiles keep most of that gain
// (the scatter 3 us slower per step than with 16) and halve the rows the
// plan walks (8 us faster).
constexpr uint32_t kChunkTiles = 32;

struct LargeSeg {
    uint32_t start, len, shift, src;
};

// The two alternating sets of an MSD level's buffers (large-segment list and
// digit histogram rows; level L reads set L & 1 and fills set (L + 1) & 1).
// With dev_level the level index is read on the device (ctr[kCtrLevel]), so a
// level's launches are the same for every level (one graph body that loops);
// otherwise every launch works on set 0.
// (Kernels select a set with a conditional, not by indexing with the level
// parity: a parameter array indexed at run time is copied to local memory.)
struct LevelRefs {
    LargeSeg *large[2];
    uint32_t *hist[2];
    uint32_t *ctr;
    int dev_level;
    int hist0_ready;   // level 0's histogram was counted before the sort (by the stitch)
    // Per large segment, its first histogram row (chunk), prefix-summed by
    // level_prefix_kernel; NULL: one row and one look-back chain per segment.
    uint32_t *chunk_prefix;
    // With hist0_ready: level 0's per-chunk histogram rows as the stitch
    // counted them, and after them the segment's total row (msd_plan reads
    // them and writes the bases to hist[0]).
    const uint32_t *top_hist;
};

__host__ __device__ __forceinline__ uint32_t seg_chunks(uint32_t len, uint32_t tile_rows)
{
    const uint32_t tiles = (len + tile_rows - 1) / tile_rows;
    return (tiles + kChunkTiles - 1) / kChunkTiles;
}

// Index of the level whose launches are running (level_prefix_kernel has
// already advanced the counter for it).
__device__ __forceinline__ uint32_t running_level(const LevelRefs &r)
{
    return r.dev_level ? *(volatile const uint32_t *)&r.ctr[kCtrLevel] - 1u : 0u;
}

template <typename K>
struct Bufs {
    K *k0, *k1;
    uint32_t *v0, *v1;
    const K *ext_bank;
    const uint32_t *ext_order;   // NULL: iota
};

template <typename K>
__device__ __forceinline__ void load_kv(const Bufs<K> &b, uint32_t src, uint64_t i, K &k, uint32_t &v)
{
    if (src == kSrcExt) {
        if (b.ext_order) {
            v = b.ext_order[i];
            k = b.ext_bank[v];
        } else {
            v = (uint32_t)i;
            k = b.ext_bank[i];
        }
    } else if (src == kSrcBuf1) {
        k = b.k1[i];
        v = b.v1[i];
    } else {
        k = b.k0[i];
        v = b.v0[i];
    }
}

template <typename K>
__device__ __forceinline__ K load_k(const Bufs<K> &b, uint32_t src, uint64_t i)
{
    if (src == kSrcExt) return b.ext_order ? b.ext_bank[b.ext_order[i]] : b.ext_bank[i];
    return src == kSrcBuf1 ? b.k1[i] : b.k0[i];
}

// A segment's rows into registers: warp-striped positions wbase + j*32 + lane
// (j < steps, position < len); the source switch is taken once per segment.
template <typename K, int IT>
__device__ __forceinline__ void load_rows(const Bufs<K> &b, uint32_t src, uint32_t start, uint32_t len, uint32_t steps,
                                          uint32_t wbase, K (&key)[IT], uint32_t (&val)[IT])
{
    const uint32_t lane = threadIdx.x & 31;
    if (src == kSrcExt && b.ext_order) {
        const uint32_t *os = b.ext_order + start;
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            val[j] = (j < (int)steps && p < len) ? os[p] : 0u;
        }
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            key[j] = (j < (int)steps && p < len) ? b.ext_bank[val[j]] : K(0);
        }
    } else if (src == kSrcExt) {
        const K *ks = b.ext_bank + start;
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            const bool ok = j < (int)steps && p < len;
            key[j] = ok ? ks[p] : K(0);
            val[j] = start + p;
        }
    } else {
        const K *ks = (src == kSrcBuf1 ? b.k1 : b.k0) + start;
        const uint32_t *vs = (src == kSrcBuf1 ? b.v1 : b.v0) + start;
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            const bool ok = j < (int)steps && p < len;
            key[j] = ok ? ks[p] : K(0);
            val[j] = ok ? vs[p] : 0u;
        }
    }
}

__device__ __forceinline__ uint2 pack_local(uint32_t start, uint32_t len, uint32_t shift, uint32_t src)
{
    return make_uint2(start, len | (shift << 16) | (src << 24));
}

struct Lists {
    uint2 *t, *t32, *a, *b1, *b2, *c1, *c1b, *c2, *c3;
    uint32_t cap_t32;      // kCapT32 for keys of <= 4 bytes, else 0 (17..32 rows go to the warp tier)
    LargeSeg *copy;        // segments that only need to reach BUF0, <= kCopySplit rows (warp each)
    LargeSeg *copy_large;  // the same, larger: copied by tiles across the grid
    uint32_t local_max;   // segments above this size take the MSD levels (tuned, <= kCapLocal)
};

// Route a segment (child or initial) to its tier.  Segments that need no
// sorting (one row, or no key bits left) only need to reach BUF0.
// A slot in the list whose counter is ctr[which]: the active lanes of a warp
// that go to the same list take their slots with one atomicAdd (children of
// one segment mostly share a tier, so the counters are hot addresses).
__device__ __forceinline__ uint32_t alloc_slot(uint32_t *ctr, int which)
{
    const uint32_t mask = __activemask();
    const uint32_t peers = __match_any_sync(mask, which);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(&ctr[which], (uint32_t)__popc(peers));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(peers & lanemask_lt());
}

// A large segment gets its next-level histogram row zeroed here when
// hist_out is given (the round's initial segments); the children of a radix
// level get theirs zeroed by that level's scatter grid, coalesced.
__device__ __forceinline__ int route_segment(uint32_t start, uint32_t len, uint32_t shift, uint32_t src,
                                             uint32_t *ctr, int large_ctr, LargeSeg *large_out, const Lists &L,
                                             uint32_t *hist_out)
{
    if (len == 0) return -1;
    int which;
    if (len == 1 || shift == 0) {
        if (src == kSrcBuf0) return -1;   // already in place
        which = len > kCopySplit ? kCtrCopyLarge : kCtrCopy;
    } else if (len > L.local_max) {
        which = large_ctr;
    } else if (len <= (uint32_t)kCapT) {
        which = kCtrLocalT;
    } else if (len <= L.cap_t32) {
        which = kCtrLocalT32;
    } else if (len <= (uint32_t)kCapA) {
        which = kCtrLocalA;
    } else if (len <= (uint32_t)kCapB1) {
        which = kCtrLocalB1;
    } else if (len <= (uint32_t)kCapB2) {
        which = kCtrLocalB2;
    } else if (len <= (uint32_t)kCapC1) {
        which = kCtrLocalC1;
    } else if (len <= (uint32_t)kCapC1b) {
        which = kCtrLocalC1b;
    } else if (len <= (uint32_t)kCapC2) {
        which = kCtrLocalC2;
    } else if (len <= (uint32_t)kCapC3) {
        which = kCtrLocalC3;
    } else {
        which = large_ctr;
    }
    const uint32_t slot = alloc_slot(ctr, which);
    const uint2 e = pack_local(start, len, shift, src);
    switch (which) {
    case kCtrCopyLarge: L.copy_large[slot] = LargeSeg{start, len, 0, src}; break;
    case kCtrCopy: L.copy[slot] = LargeSeg{start, len, 0, src}; break;
    case kCtrLocalT: L.t[slot] = e; break;
    case kCtrLocalT32: L.t32[slot] = e; break;
    case kCtrLocalA: L.a[slot] = e; break;
    case kCtrLocalB1: L.b1[slot] = e; break;
    case kCtrLocalB2: L.b2[slot] = e; break;
    case kCtrLocalC1: L.c1[slot] = e; break;
    case kCtrLocalC1b: L.c1b[slot] = e; break;
    case kCtrLocalC2: L.c2[slot] = e; break;
    case kCtrLocalC3: L.c3[slot] = e; break;
    default: {
        large_out[slot] = LargeSeg{start, len, shift, src};
        if (hist_out) {
            uint4 *row = reinterpret_cast<uint4 *>(hist_out + (uint64_t)slot * kRadix);
#pragma unroll 4
            for (int i = 0; i < kRadix / 4; ++i) row[i] = make_uint4(0, 0, 0, 0);
        }
    }
    }
    return which;
}

// ---------------------------------------------------------------------------
// classification of the round's initial segments
// ---------------------------------------------------------------------------
template <typename K>
__global__ void classify_kernel(Bufs<K> b, const uint32_t *__restrict__ seg_start, const uint32_t *d_nseg,
                                uint64_t n, uint32_t key_bits, uint32_t *ctr, LargeSeg *large0, Lists lists,
                                const uint32_t *top_hist, const uint32_t *d_key_bits, const uint32_t *d_in_order)
{
    kernel_prologue();
    if (d_key_bits) key_bits = min(key_bits, *d_key_bits);
    if (d_in_order && *d_in_order) key_bits = 0;   // every segment is in order: copy only
    if (!seg_start && top_hist && n > lists.local_max) {
        // round 0 over the whole array with its first-level histogram already
        // counted (level 0's msd_plan reads the stitch's rows): the one large
        // segment
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctr[kCtrLarge0] = 1;
            large0[0] = LargeSeg{0, (uint32_t)n, key_bits, kSrcExt};
        }
        return;
    }
    const uint32_t nseg = seg_start ? *d_nseg : 1u;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        const uint32_t start = seg_start ? seg_start[s] : 0u;
        const uint32_t end = seg_start ? seg_start[s + 1] : (uint32_t)n;
        const uint32_t len = end - start;
        if (len == 1) {
            // A one-row segment keeps its position: copy it straight to BUF0.
            K k;
            uint32_t v;
            load_kv(b, kSrcExt, start, k, v);
            b.k0[start] = k;
            b.v0[start] = v;
            continue;
        }
        // (level 0's histogram rows are zeroed by its level_prefix_kernel)
        route_segment(start, len, key_bits, kSrcExt, ctr, kCtrLarge0, large0, lists, nullptr);
    }
}

// ---------------------------------------------------------------------------
// MSD level kernels (large segments)
// ---------------------------------------------------------------------------
// Exclusive prefix of the tile counts of the level's large segments (one CTA).
// Also resets the level's counters (tile counter, rows moved, next-level
// count) so that no separate memsets are needed.
__device__ __forceinline__ void tile_prefix_body(const LargeSeg *segs, uint32_t nseg, uint32_t *tile_prefix,
                                                 uint32_t tile_rows, bool chunks = false)
{
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < nseg; base += blockDim.x) {
        const uint32_t s = base + threadIdx.x;
        const uint32_t c = s >= nseg ? 0u
                           : chunks  ? seg_chunks(segs[s].len, tile_rows)
                                     : (segs[s].len + tile_rows - 1) / tile_rows;
        uint32_t incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane_id() >= o) incl += y;
        }
        if (lane_id() == 31) warp_sums[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint32_t v = threadIdx.x < blockDim.x / 32 ? warp_sums[threadIdx.x] : 0u;
            uint32_t vi = v;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xFFFFFFFFu, vi, o);
                if ((int)threadIdx.x >= o) vi += y;
            }
            warp_sums[threadIdx.x] = vi - v;
        }
        __syncthreads();
        const uint32_t excl = carry + warp_sums[threadIdx.x >> 5] + incl - c;
        if (s < nseg) tile_prefix[s] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_prefix[nseg] = carry;
}

__global__ void __launch_bounds__(1024) tile_prefix_kernel(const LargeSeg *segs, const uint32_t *d_nseg,
                                                           uint32_t *tile_prefix, uint32_t *reset, uint32_t tile_rows)
{
    kernel_prologue();
    if (threadIdx.x == 0) *reset = 0;
    tile_prefix_body(segs, *d_nseg, tile_prefix, tile_rows);
}

// First launch of an MSD level: tile prefix of the level's large segments,
// resets of the level's counters, and (device-side levels) the level index
// advanced for the level's other launches.
__global__ void __launch_bounds__(1024) level_prefix_kernel(LevelRefs r, uint32_t *tile_prefix, uint32_t tile_rows)
{
    kernel_prologue();
    const uint32_t lvl = r.dev_level ? r.ctr[kCtrLevel] : 0u;
    const uint32_t cur = lvl & 1u, nxt = cur ^ 1u;
    const uint32_t nseg = r.ctr[kCtrLarge0 + cur];
    __syncthreads();   // every thread has read the level index before it advances
    if (threadIdx.x == 0) {
        r.ctr[kCtrLarge0 + nxt] = 0;
        r.ctr[kCtrChunks0 + nxt] = 0;
        r.ctr[kCtrMsdTile] = 0;
        r.ctr[kCtrMoved] = 0;
        if (r.dev_level) r.ctr[kCtrLevel] = lvl + 1;
    }
    const LargeSeg *segs = cur ? r.large[1] : r.large[0];
    tile_prefix_body(segs, nseg, tile_prefix, tile_rows);
    if (r.chunk_prefix) {
        tile_prefix_body(segs, nseg, r.chunk_prefix, tile_rows, true);
        if (lvl == 0 && !r.hist0_ready) {
            // level 0's histogram rows start at zero (a level's scatter zeroes
            // the next level's rows)
            __syncthreads();
            const uint64_t words = (uint64_t)r.chunk_prefix[nseg] * (kRadix / 4);
            uint4 *h = reinterpret_cast<uint4 *>(cur ? r.hist[1] : r.hist[0]);
            for (uint64_t i = threadIdx.x; i < words; i += blockDim.x) h[i] = make_uint4(0, 0, 0, 0);
        }
    }
}


// The segment of tile t (tile_prefix[s] <= t < tile_prefix[s + 1]), found by
// a whole warp (t the same in every lane): each round the 32 lanes probe 32
// evenly spaced prefixes, so the range shrinks 32-fold per dependent load (two
// rounds for 1,024 segments) instead of 2-fold as in a binary search.
__device__ __forceinline__ uint32_t find_segment_warp(const uint32_t *tile_prefix, uint32_t nseg, uint32_t t)
{
    uint32_t lo = 0, hi = nseg;  // tile_prefix[lo] <= t < tile_prefix[hi]
    const uint32_t lane = lane_id();
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t m = lo + lane * step;
        // the prefixes do not decrease: the lanes whose probe is <= t are a
        // prefix of the warp, and lane 0 (probing lo) is one of them
        const bool le = m < hi && tile_prefix[m] <= t;
        const uint32_t c = __popc(__ballot_sync(0xFFFFFFFFu, le));
        lo += (c - 1) * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// Top-digit histogram of every large segment.  A block takes a contiguous run
// of tiles; each thread issues all of a tile's loads before counting (up to 16
// in flight), and each warp counts into its own shared sub-histogram so that
// skewed digits do not serialize the whole block on one counter.
template <typename K>
__global__ void __launch_bounds__(kNtM, kHistCtas) msd_hist_kernel(Bufs<K> b, LevelRefs r, const uint32_t *tile_prefix,
                                                        uint32_t tile_rows)
{
    kernel_prologue();
    constexpr int NW = kNtM / 32;
    constexpr int MAXJ = 16;   // tile_rows <= 16 * kNtM
    __shared__ uint32_t sh[NW][kRadix];
    const uint32_t lvl = running_level(r);
    if (lvl == 0 && r.hist0_ready) return;
    const uint32_t cur = lvl & 1u;
    const LargeSeg *segs = (cur ? r.large[1] : r.large[0]);
    uint32_t *hist = (cur ? r.hist[1] : r.hist[0]);
    const uint32_t nseg = r.ctr[kCtrLarge0 + cur];
    if (nseg == 0) return;
    const uint32_t T = tile_prefix[nseg];
    const int warp = threadIdx.x >> 5;
    // a contiguous run of tiles per block; the per-warp counts are added to
    // the segment's histogram when the run moves to the next segment (every
    // large segment has at least one tile) and at its end
    const uint32_t per = (T + gridDim.x - 1) / gridDim.x;
    const uint32_t t0 = blockIdx.x * per;
    const uint32_t t1 = min(T, t0 + per);
    if (t0 >= T) return;
    for (int d = threadIdx.x; d < NW * kRadix; d += blockDim.x) (&sh[0][0])[d] = 0;
    uint32_t s = find_segment_warp(tile_prefix, nseg, t0);
    LargeSeg sg = segs[s];
    uint32_t sfirst = tile_prefix[s], snext = tile_prefix[s + 1];
    // the histogram row of the tiles counted so far: the segment's, or its
    // chunk's when the level cuts segments into chunks
    auto row_of = [&](uint32_t seg, uint32_t k) -> uint32_t {
        return r.chunk_prefix ? r.chunk_prefix[seg] + k / kChunkTiles : seg;
    };
    uint32_t row = row_of(s, t0 - sfirst);
    auto flush = [&]() {
        __syncthreads();
        for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
            uint32_t c = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                c += sh[w][d];
                sh[w][d] = 0;
            }
            if (c) atomicAdd(&hist[(uint64_t)row * kRadix + d], c);
        }
        __syncthreads();
    };
    __syncthreads();
    for (uint32_t t = t0; t < t1; ++t) {
        if (t >= snext) {   // every large segment has a tile: the next tile starts the next segment
            ++s;
            sg = segs[s];
            sfirst = snext;
            snext = tile_prefix[s + 1];
        }
        const uint32_t k = t - sfirst;
        const uint32_t trow = row_of(s, k);
        if (trow != row) {
            flush();
            row = trow;
        }
        const uint32_t width = sg.shift < (uint32_t)kRadixBits ? sg.shift : (uint32_t)kRadixBits;
        const uint32_t lo = sg.shift - width;
        const uint64_t beg = (uint64_t)sg.start + (uint64_t)k * tile_rows;
        const uint64_t end = min((uint64_t)sg.start + sg.len, beg + tile_rows);
        K key[MAXJ];
#pragma unroll
        for (int j = 0; j < MAXJ; ++j) {
            const uint64_t i = beg + threadIdx.x + (uint64_t)j * kNtM;
            if (i < end) key[j] = load_k(b, sg.src, i);
        }
#pragma unroll
        for (int j = 0; j < MAXJ; ++j) {
            const uint64_t i = beg + threadIdx.x + (uint64_t)j * kNtM;
            if (i < end) atomicAdd(&sh[warp][digit_of(key[j], lo, width)], 1u);
        }
    }
    flush();
}

// Per large segment: exclusive digit offsets, skip detection, children.
// With chunks, a segment's digit counts are the sums of its chunks' rows, and
// each chunk's row becomes its digit bases: the segment's offset of the digit
// plus the digit's rows in the segment's earlier chunks.  kPlanThreads threads
// per segment: kPlanThreads / kRadix of them per digit, each summing (then
// rewriting) a contiguous share of the chunk rows with kPlanLoads loads in
// flight, so that a segment of a hundred chunks costs a few round trips.
// (1024 threads per segment walk long segments faster, but four times fewer
// segments are planned at once: slower in all.)
constexpr int kPlanThreads = 256;
constexpr int kPlanLoads = 16;
constexpr int kPlanHelpers = 8;   // CTAs writing level 0's chunk bases beside the segment's CTA
static_assert(kRadix % kPlanHelpers == 0 && kPlanThreads % (kRadix / kPlanHelpers) == 0 &&
              kPlanThreads / (kRadix / kPlanHelpers) <= 32, "plan helper layout");

__global__ void __launch_bounds__(kPlanThreads) msd_plan_kernel(LevelRefs r, Lists lists, bool emit_children = true,
                                                                uint32_t tile_rows = 0)
{
    kernel_prologue();
    constexpr int NQ = kPlanThreads / kRadix;   // threads per digit
    __shared__ uint32_t cnt[kRadix];
    __shared__ uint32_t part[NQ][kRadix];
    __shared__ uint32_t tmp[kPlanThreads / 32 + 1];
    __shared__ uint32_t s_skip;
    const uint32_t lvl = running_level(r);
    const uint32_t cur = lvl & 1u, nxt = cur ^ 1u;
    LargeSeg *segs = (cur ? r.large[1] : r.large[0]);
    uint32_t *hist = (cur ? r.hist[1] : r.hist[0]);
    // the counts: this level's rows, or at level 0 the stitch's
    const uint32_t *counts = (lvl == 0 && r.hist0_ready && r.top_hist) ? r.top_hist : hist;
    uint32_t *ctr = r.ctr;
    const int next_large_ctr = kCtrLarge0 + (int)nxt;
    LargeSeg *large_next = (nxt ? r.large[1] : r.large[0]);
    const uint32_t nseg = ctr[kCtrLarge0 + cur];
    const uint32_t d = threadIdx.x % kRadix;
    const uint32_t q4 = threadIdx.x / kRadix;
    // Level 0 counted by the stitch: one segment with its totals in the last
    // row.  CTA 0 plans the segment; CTAs 1..kPlanHelpers write the chunk
    // bases, each for kRadix / kPlanHelpers digits with kPlanThreads /
    // (kRadix / kPlanHelpers) threads per digit, each over a share of the rows
    // (a scan across the digit's threads joins the shares).
    const bool split0 = counts == r.top_hist && r.chunk_prefix != nullptr;
    if (split0 && blockIdx.x >= 1 && blockIdx.x <= (unsigned)kPlanHelpers && nseg == 1) {
        constexpr uint32_t DPB = kRadix / kPlanHelpers;        // digits per helper CTA
        constexpr uint32_t TPD = kPlanThreads / DPB;           // threads per digit (a power of two <= 32)
        const uint32_t nrows = r.chunk_prefix[1];
        cnt[d] = q4 == 0 ? counts[(uint64_t)nrows * kRadix + d] : 0u;
        uint32_t total;
        block_exclusive_scan_radix<kPlanThreads>(cnt, tmp, &total);
        const uint32_t dd = (blockIdx.x - 1) * DPB + threadIdx.x / TPD;
        const uint32_t sub = threadIdx.x % TPD;
        const uint32_t per = (nrows + TPD - 1) / TPD;
        const uint32_t qa = min(nrows, sub * per), qb = min(nrows, qa + per);
        uint32_t c = 0;
        for (uint32_t q = qa; q < qb; q += kPlanLoads) {
            uint32_t v[kPlanLoads];
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) v[j] = q + j < qb ? counts[(uint64_t)(q + j) * kRadix + dd] : 0u;
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) c += v[j];
        }
        // exclusive scan of the shares across the digit's TPD lanes
        uint32_t incl = c;
#pragma unroll
        for (uint32_t o = 1; o < TPD; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o, TPD);
            if (sub >= o) incl += y;
        }
        uint32_t run = cnt[dd] + incl - c;
        for (uint32_t q = qa; q < qb; q += kPlanLoads) {
            uint32_t v[kPlanLoads];
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) v[j] = q + j < qb ? counts[(uint64_t)(q + j) * kRadix + dd] : 0u;
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) {
                if (q + j < qb) hist[(uint64_t)(q + j) * kRadix + dd] = run;
                run += v[j];
            }
        }
        return;
    }
    for (uint32_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        const LargeSeg sg = segs[s];
        const uint32_t r0 = r.chunk_prefix ? r.chunk_prefix[s] : s;
        const uint32_t r1 = r.chunk_prefix ? r.chunk_prefix[s + 1] : s + 1;
        // this thread's share of the rows
        const uint32_t per = (r1 - r0 + NQ - 1) / NQ;
        const uint32_t qa = min(r1, r0 + q4 * per), qb = min(r1, qa + per);
        uint32_t c = 0;
        if (counts == r.top_hist) {
            // the stitch's rows end with the (one) segment's total
            if (q4 == 0) c = counts[(uint64_t)r1 * kRadix + d];
        } else {
            for (uint32_t q = qa; q < qb; q += kPlanLoads) {
                uint32_t v[kPlanLoads];
#pragma unroll
                for (int j = 0; j < kPlanLoads; ++j) v[j] = q + j < qb ? counts[(uint64_t)(q + j) * kRadix + d] : 0u;
#pragma unroll
                for (int j = 0; j < kPlanLoads; ++j) c += v[j];
            }
        }
        part[q4][d] = c;
        if (threadIdx.x == 0) s_skip = 0;
        __syncthreads();
        uint32_t tot = 0;
        if (q4 == 0) {
#pragma unroll
            for (int j = 0; j < NQ; ++j) tot += part[j][d];
            cnt[d] = tot;
            if (tot == sg.len) s_skip = 1;   // every row has this digit: the pass is the identity
        }
        uint32_t total;
        block_exclusive_scan_radix<kPlanThreads>(cnt, tmp, &total);
        const uint32_t off = cnt[d];
        // this share's first base: the digit's offset plus the earlier shares' rows
        uint32_t run = off;
        for (uint32_t j = 0; j < q4; ++j) run += part[j][d];
        // (with split0 and one segment the helper CTAs write the bases)
        for (uint32_t q = qa; q < (split0 && nseg == 1 ? qa : qb); q += kPlanLoads) {
            uint32_t v[kPlanLoads];
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) v[j] = q + j < qb ? counts[(uint64_t)(q + j) * kRadix + d] : 0u;
#pragma unroll
            for (int j = 0; j < kPlanLoads; ++j) {
                if (q + j < qb) hist[(uint64_t)(q + j) * kRadix + d] = run;
                run += v[j];
            }
        }
        const bool skip = s_skip != 0;
        const uint32_t width = sg.shift < (uint32_t)kRadixBits ? sg.shift : (uint32_t)kRadixBits;
        const uint32_t child_shift = sg.shift - width;
        const uint32_t child_src = skip ? sg.src : (sg.src == kSrcBuf1 ? kSrcBuf0 : kSrcBuf1);
        if (q4 == 0 && emit_children && tot > 0) {
            // (the next level's histogram rows are zeroed by the scatter grid)
            const int which = route_segment(sg.start + off, tot, child_shift, child_src, ctr, next_large_ctr,
                                            large_next, lists, nullptr);
            if (r.chunk_prefix) {
                // the large children's chunks, one atomic per warp
                const uint32_t mask = __activemask();
                const uint32_t add = __reduce_add_sync(mask, which == next_large_ctr ? seg_chunks(tot, tile_rows)
                                                                                     : 0u);
                if ((int)lane_id() == __ffs(mask) - 1 && add) atomicAdd(&ctr[kCtrChunks0 + nxt], add);
            }
        }
        if (threadIdx.x == 0 && skip) segs[s].src = sg.src | kSkipBit;
        if (threadIdx.x == 0 && !skip) atomicAdd(&ctr[kCtrMoved], sg.len);
        __syncthreads();
    }
}

// Resident CTAs of the scatter per SM (the launch bound and the grid).
constexpr int msd_ctas_per_sm(int it) { return it >= 16 ? kMsdCtas16 : 4; }

template <typename K, int IT>
struct MsdSmem {
    uint32_t whist[kNtM / 32][kRadix];
    uint32_t total[kRadix];
    uint32_t doff[kRadix];       // tile-local exclusive digit offsets
    uint32_t gdst[kRadix];       // global destination base per digit (mod 2^32; rows < 2^32)
    uint32_t tmp[kNtM / 32 + 1];
    uint32_t tile, seg;
    K keys[kNtM * IT];
    uint32_t vals[kNtM * IT];
    static_assert(kNtM * IT >= (kNtM / 32) * kRadix, "the peer words of kRankOr fit in vals");
};

template <typename K, int RANK, int IT>
__global__ void __launch_bounds__(kNtM, msd_ctas_per_sm(IT)) msd_scatter_kernel(Bufs<K> b, LevelRefs r,
                                                           const uint32_t *tile_prefix, unsigned long long *lookback,
                                                           uint32_t epoch_base, int *status,
                                                           cudaGraphConditionalHandle more, uint32_t levels)
{
    kernel_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MsdSmem<K, IT> &sm = *reinterpret_cast<MsdSmem<K, IT> *>(smem_raw);
    constexpr uint32_t kTileM = kNtM * IT;
    const uint32_t lvl = running_level(r);
    const uint32_t cur = lvl & 1u;
    const LargeSeg *segs = (cur ? r.large[1] : r.large[0]);
    const uint32_t *offs = (cur ? r.hist[1] : r.hist[0]);
    uint32_t *tile_counter = &r.ctr[kCtrMsdTile];
    const uint32_t epoch = epoch_base + lvl;
    const uint32_t nseg = r.ctr[kCtrLarge0 + cur];
    // Inside a graph, the level loop goes on while the next level has large
    // segments (msd_plan has counted them before this launch).
    const uint32_t nnext = r.ctr[kCtrLarge0 + (cur ^ 1u)];
    if (more && blockIdx.x == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(more, (nnext > 0 && lvl + 1 < levels) ? 1u : 0u);
    {
        // the histogram rows of the next level's large segments (or of their
        // chunks, counted by this level's plan) start at zero (the rows held
        // this level's predecessor's offsets, which nothing reads any more)
        uint4 *h = reinterpret_cast<uint4 *>(cur ? r.hist[0] : r.hist[1]);
        const uint32_t rows_next = r.chunk_prefix ? r.ctr[kCtrChunks0 + (cur ^ 1u)] : nnext;
        const uint64_t words = (uint64_t)rows_next * (kRadix / 4);
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < words;
             i += (uint64_t)gridDim.x * blockDim.x)
            h[i] = make_uint4(0, 0, 0, 0);
    }
    if (nseg == 0) return;
    const uint32_t T = tile_prefix[nseg];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0) sm.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= T) break;
        const uint32_t s = find_segment_warp(tile_prefix, nseg, t);
        const LargeSeg sg = segs[s];
        if (sg.src & kSkipBit) {
            __syncthreads();
            continue;
        }
        const uint32_t k = t - tile_prefix[s];
        // the tile's histogram row and its place in its look-back chain
        const uint32_t row = r.chunk_prefix ? r.chunk_prefix[s] + k / kChunkTiles : s;
        const uint32_t kc = r.chunk_prefix ? k % kChunkTiles : k;
        const uint32_t width = sg.shift < (uint32_t)kRadixBits ? sg.shift : (uint32_t)kRadixBits;
        const uint32_t lo = sg.shift - width;
        const uint64_t tbeg = (uint64_t)sg.start + (uint64_t)k * kTileM;
        const uint64_t send = (uint64_t)sg.start + sg.len;
        const uint32_t cnt = (uint32_t)min((uint64_t)kTileM, send - tbeg);
        // kRankOr's per-warp peer words live in the vals staging area, which
        // is free until the ranks are known
        uint32_t *peerw = &sm.vals[warp * kRadix];
        for (int d = lane; d < kRadix; d += 32) {
            sm.whist[warp][d] = 0;
            if constexpr (RANK == kRankOr) peerw[d] = 0;
        }
        __syncwarp();

        K key[IT];
        uint32_t val[IT];
        uint32_t rd[IT];   // rank in the warp (low 16 bits) | digit << 16
        const uint32_t wbase = warp * (IT * 32);
        load_rows<K, IT>(b, sg.src, (uint32_t)tbeg, cnt, IT, wbase, key, val);
        if (cnt == kTileM && width == (uint32_t)kRadixBits) {
            // a whole tile and a whole digit (the common case): no lane checks
#pragma unroll
            for (int j = 0; j < IT; ++j) {
                const uint32_t d = (uint32_t)((uint64_t)key[j] >> lo) & (uint32_t)(kRadix - 1);
                if constexpr (RANK == kRankOr)
                    rd[j] = wlms_rank_or(d, true, sm.whist[warp], peerw) | (d << 16);
                else
                    rd[j] = wlms_rank_full<RANK>(d, sm.whist[warp]) | (d << 16);
            }
        } else {
#pragma unroll
            for (int j = 0; j < IT; ++j) {
                const uint32_t p = wbase + j * 32 + lane;
                const uint32_t d = digit_of(key[j], lo, width);
                if constexpr (RANK == kRankOr)
                    rd[j] = wlms_rank_or(d, p < cnt, sm.whist[warp], peerw) | (d << 16);
                else
                    rd[j] = wlms_rank<RANK>(d, p < cnt, sm.whist[warp], width) | (d << 16);
            }
        }
        __syncthreads();
        // per digit: exclusive over warps, tile total
        for (int d = threadIdx.x; d < kRadix; d += kNtM) {
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < kNtM / 32; ++w) {
                const uint32_t c = sm.whist[w][d];
                sm.whist[w][d] = run;
                run += c;
            }
            sm.total[d] = run;
            sm.doff[d] = run;
            unsigned long long *mine = &lookback[(uint64_t)t * kRadix + d];
            st_volatile_u64(mine, lb_word(epoch, kc == 0 ? kFlagInclusive : kFlagAggregate, run));
        }
        __syncthreads();
        uint32_t tot;
        block_exclusive_scan_radix<kNtM>(sm.doff, sm.tmp, &tot);
        // decoupled look-back along the chunk's tiles
        for (int d = threadIdx.x; d < kRadix; d += kNtM) {
            uint32_t excl = 0;
            if (kc > 0) {
                int64_t p = (int64_t)t - 1;
                for (;;) {
                    const unsigned long long w = lb_wait(&lookback[(uint64_t)p * kRadix + d], epoch, status);
                    excl += (uint32_t)w;
                    if (((uint32_t)(w >> 32) & 3u) == kFlagInclusive) break;
                    --p;
                }
                st_volatile_u64(&lookback[(uint64_t)t * kRadix + d],
                                lb_word(epoch, kFlagInclusive, excl + sm.total[d]));
            }
            const uint32_t dof = sm.doff[d];
            sm.gdst[d] = sg.start + offs[(uint64_t)row * kRadix + d] + excl - dof;   // wraps; + slot is in range
            // the warps' exclusive counts become tile positions
#pragma unroll
            for (int w = 0; w < kNtM / 32; ++w) sm.whist[w][d] += dof;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            if (p < cnt) {
                const uint32_t pos = sm.whist[warp][rd[j] >> 16] + (rd[j] & 0xFFFFu);
                sm.keys[pos] = key[j];
                sm.vals[pos] = val[j];
            }
        }
        __syncthreads();
        K *dk = (sg.src == kSrcBuf1) ? b.k0 : b.k1;
        uint32_t *dv = (sg.src == kSrcBuf1) ? b.v0 : b.v1;
        for (uint32_t i = threadIdx.x; i < cnt; i += kNtM) {
            const K kk = sm.keys[i];
            const uint32_t o = sm.gdst[digit_of(kk, lo, width)] + i;
            dk[o] = kk;
            dv[o] = sm.vals[i];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// local tiers
// ---------------------------------------------------------------------------
// Block-per-segment stable sort over key bits [0, shift).  One HBM read and
// one HBM write per row; everything else in shared memory.
//
// Fast path (bucket_rank_sort): the bits in which the segment's keys differ
// are found by an OR/AND reduction; rows are bucketed by the top
// ceil(log2(len)) of those bits (about one row per bucket) with shared-memory
// atomics, in no particular order inside a bucket; each row's final place is
// then its bucket's start plus the number of rows of the bucket that sort
// before it by (key, position in the segment).  Ties are decided by the
// position, so the result is the stable order although the bucketing is not.
//
// Fallback, when some bucket holds more than kBucketMax rows (heavily
// repeated keys):
//   1. one stable split on the top digit (bits [shift-8, shift)), ranked by
//      warp-level multi-split: rows land in 256 buckets in key order;
//   2. if every bucket holds <= kCountRankMax rows, each row's final place is
//      bucket start + the number of rows of its bucket that sort before it
//      (smaller key, or equal key and earlier position): a short loop over
//      the bucket with broadcast shared-memory reads, no further passes;
//   3. otherwise (skewed keys) LSD passes over bits [0, shift-8) and a last
//      pass on the top digit finish the sort from the split order.
// Every step is stable, so ties keep their input order.
constexpr uint32_t kCountRankMax = 64;
constexpr uint32_t kBucketMax = 64;

constexpr int pow2_ceil(int x)
{
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

template <typename K, int NT, int IT>
struct BucketSmem {
    unsigned long long cs[NT * IT];   // compound keys, bucketed
    uint32_t vals[NT * IT];
    uint32_t off[pow2_ceil(NT * IT) + 1];   // per bucket: count -> start (up to 2^ceil(log2 len) buckets)
    uint16_t orig[NT * IT];           // position in the segment, when the compound key has no room for it
    uint32_t tmp[NT / 32 + 1];
    unsigned long long any, all;      // OR and AND of the segment's keys
    uint32_t maxb;
};

// Exclusive scan of off[0, nb) by the block (nb a power of two, at most
// NT * IT, so at most 16 * NT), also leaving the largest count in *maxb.
// Thread t scans its own run of PER = nb / NT consecutive bins (one bin each
// for the first nb threads when nb < NT), read as vectors and summed, then,
// after the runs' totals are scanned across the block, read again and written
// back as exclusive offsets (the run is not held in registers across the
// barriers).  A run of NV > 1 16-byte vectors is visited starting at vector
// (t * PER / 32) mod NV, so that the 8 threads of a shared-memory wavefront
// touch 8 different bank groups instead of 2 to 4.
template <int NT, int PER>
__device__ __forceinline__ void scan_bin_runs(uint32_t *off, uint32_t nb, uint32_t *tmp, uint32_t *maxb)
{
    constexpr int NW = NT / 32;
    constexpr int VW = PER >= 4 ? 4 : PER;   // words per vector access
    constexpr int NV = PER / VW;             // vectors per run
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t b0 = threadIdx.x * PER;
    const bool mine = b0 < nb;
    const uint32_t rot = NV > 1 ? (threadIdx.x * PER / 32) : 0u;
    auto vec_of = [&](int q) -> uint32_t { return ((uint32_t)q + rot) & (uint32_t)(NV - 1); };
    auto ld = [&](uint32_t v, uint32_t (&x)[VW]) {
        if constexpr (VW == 4) {
            const uint4 w = reinterpret_cast<const uint4 *>(off + b0)[v];
            x[0] = w.x; x[1] = w.y; x[2] = w.z; x[3] = w.w;
        } else if constexpr (VW == 2) {
            const uint2 w = reinterpret_cast<const uint2 *>(off + b0)[v];
            x[0] = w.x; x[1] = w.y;
        } else {
            x[0] = off[b0 + v];
        }
    };
    uint32_t sum = 0, mx = 0;
    if (mine) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            uint32_t x[VW];
            ld(vec_of(q), x);
#pragma unroll
            for (int i = 0; i < VW; ++i) {
                sum += x[i];
                mx = max(mx, x[i]);
            }
        }
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if (lane == 31) tmp[warp] = incl;
    if (lane == 0 && mx) atomicMax(maxb, mx);
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < NW ? tmp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < NW) tmp[lane] = wi - w;
    }
    __syncthreads();
    if (mine) {
        const uint32_t run = tmp[warp] + incl - sum;
        // the run's vectors in visiting order, with their sums
        uint32_t x[NV][VW], vs[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            ld(vec_of(q), x[q]);
            vs[q] = 0;
#pragma unroll
            for (int i = 0; i < VW; ++i) vs[q] += x[q][i];
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            // the vector's first offset: the run's plus every vector before it
            uint32_t r = run;
#pragma unroll
            for (int u = 0; u < NV; ++u) r += vec_of(u) < vec_of(q) ? vs[u] : 0u;
#pragma unroll
            for (int i = 0; i < VW; ++i) {
                const uint32_t c = x[q][i];
                x[q][i] = r;
                r += c;
            }
            const uint32_t v = vec_of(q);
            if constexpr (VW == 4) reinterpret_cast<uint4 *>(off + b0)[v] = make_uint4(x[q][0], x[q][1], x[q][2], x[q][3]);
            else if constexpr (VW == 2) reinterpret_cast<uint2 *>(off + b0)[v] = make_uint2(x[q][0], x[q][1]);
            else off[b0 + v] = x[q][0];
        }
    }
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ void block_scan_bins(uint32_t *off, uint32_t nb, uint32_t *tmp, uint32_t *maxb)
{
    switch (nb >= (uint32_t)NT ? nb / NT : 1u) {
    case 1: scan_bin_runs<NT, 1>(off, nb, tmp, maxb); break;
    case 2: scan_bin_runs<NT, 2>(off, nb, tmp, maxb); break;
    case 4: scan_bin_runs<NT, 4>(off, nb, tmp, maxb); break;
    case 8: scan_bin_runs<NT, 8>(off, nb, tmp, maxb); break;
    default: scan_bin_runs<NT, 16>(off, nb, tmp, maxb); break;
    }
}

// The fast path above.  Rows are in registers (warp w holds positions
// wbase + j*32 + lane, j < steps).  Returns false, with nothing written,
// when a bucket is too large; the caller then runs the stable fallback.
// Ends with a block barrier either way.
//
// Compound key: the key bits below `top` (the bits above are the same in
// every row), shifted left by nbits with the row's position in the low
// nbits when they fit in 64 bits, so that compound keys are all distinct and
// compare like (key, position).  Otherwise the position is kept beside it.
// A row's bucket is the top `width` bits of its compound key (about one row
// per bucket); its final place is its bucket's start plus the rows of the
// bucket with a smaller compound key.  A row alone in its bucket is in its
// place without comparisons.
template <typename K, int NT, int IT>
__device__ __forceinline__ bool bucket_rank_sort(BucketSmem<K, NT, IT> &sm, const K (&key)[IT],
                                                 const uint32_t (&val)[IT], uint32_t steps, uint32_t wbase,
                                                 uint32_t len, const Bufs<K> &b, uint32_t start)
{
    const int lane = threadIdx.x & 31;
    const uint32_t nbits = 32u - (uint32_t)__clz(len - 1u);          // ceil(log2(len)), len >= 2
    if (threadIdx.x == 0) {
        sm.any = 0ull;
        sm.all = ~0ull;
        sm.maxb = 0;
    }
    // bucket counters for any digit width up to nbits
    for (uint32_t i = threadIdx.x; i <= (1u << nbits); i += NT) sm.off[i] = 0;
    __syncthreads();
    unsigned long long any = 0ull, all = ~0ull;
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t p = wbase + j * 32 + lane;
        if (j < (int)steps && p < len) {
            any |= (unsigned long long)key[j];
            all &= (unsigned long long)key[j];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        any |= __shfl_xor_sync(0xFFFFFFFFu, any, o);
        all &= __shfl_xor_sync(0xFFFFFFFFu, all, o);
    }
    if (lane == 0) {
        atomicOr(&sm.any, any);
        atomicAnd(&sm.all, all);
    }
    __syncthreads();
    K *ko = b.k0 + start;
    uint32_t *vo = b.v0 + start;
    const unsigned long long diff = sm.any & ~sm.all;
    if (diff == 0ull) {
        // every key is the same: the segment is in order already
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            if (j < (int)steps && p < len) {
                ko[p] = key[j];
                vo[p] = val[j];
            }
        }
        __syncthreads();
        return true;
    }
    const uint32_t top = 64u - (uint32_t)__clzll((long long)diff);   // bits [0, top) differ somewhere
    const unsigned long long low = top >= 64u ? ~0ull : ((1ull << top) - 1ull);
    const unsigned long long prefix = sm.all & ~low;                 // the bits every row shares
    const bool packed = top + nbits <= 64u;
    const uint32_t sh = packed ? nbits : 0u;
    const uint32_t lo = top > nbits ? top - nbits : 0u;
    const uint32_t width = top - lo;
    const uint32_t dshift = lo + sh;                                 // bucket = compound >> dshift
    const uint32_t nb = 1u << width;
    unsigned long long c[IT];
    uint32_t slot[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t p = wbase + j * 32 + lane;
        if (j < (int)steps && p < len) {
            c[j] = (((unsigned long long)key[j] & low) << sh) | (packed ? p : 0u);
            slot[j] = atomicAdd(&sm.off[(uint32_t)(c[j] >> dshift)], 1u);
        }
    }
    __syncthreads();
    block_scan_bins<NT>(sm.off, nb, sm.tmp, &sm.maxb);
    if (sm.maxb > kBucketMax) {
        __syncthreads();
        return false;   // uniform across the block
    }
    // rows land bucketed; each keeps its bucket's start and size (start | size << 16)
    uint32_t bk[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t p = wbase + j * 32 + lane;
        bk[j] = 0;
        if (j < (int)steps && p < len) {
            const uint32_t bi = (uint32_t)(c[j] >> dshift);
            const uint32_t bs = sm.off[bi];
            const uint32_t be = bi + 1 < nb ? sm.off[bi + 1] : len;
            const uint32_t pos = bs + slot[j];
            bk[j] = bs | ((be - bs) << 16);
            sm.cs[pos] = c[j];
            sm.vals[pos] = val[j];
            if (!packed) sm.orig[pos] = (uint16_t)p;
        }
    }
    __syncthreads();
    // a row alone in its bucket is in its place; the others count the rows of
    // their bucket that sort before them (by compound key, then position)
    uint32_t fin[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t bs = bk[j] & 0xFFFFu, bn = bk[j] >> 16;
        uint32_t r = 0;
        if (bn > 1) {
            if (packed) {
                for (uint32_t q = 0; q < bn; ++q) r += sm.cs[bs + q] < c[j];
            } else {
                const uint32_t o = wbase + j * 32 + lane;
                for (uint32_t q = 0; q < bn; ++q) {
                    const unsigned long long cq = sm.cs[bs + q];
                    r += (cq < c[j]) | ((cq == c[j]) & ((uint32_t)sm.orig[bs + q] < o));
                }
            }
        }
        fin[j] = bs + r;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        if ((bk[j] >> 16) > 1) {
            sm.cs[fin[j]] = c[j];
            sm.vals[fin[j]] = val[j];
        }
    }
    __syncthreads();
    // every load of this segment is done (barriers above) before the first
    // store into BUF0, which may alias the EXT oids of the range
    for (uint32_t p = threadIdx.x; p < len; p += NT) {
        ko[p] = (K)(prefix | (sm.cs[p] >> sh));
        vo[p] = sm.vals[p];
    }
    __syncthreads();
    return true;
}

template <typename K, int NT, int IT>
struct BlockSmem {
    uint32_t whist[NT / 32][kRadix];
    uint32_t doff[kRadix];
    uint32_t cnt[kRadix];
    uint32_t tmp[NT / 32 + 1];
    uint32_t flag;
    uint32_t maxb;
    K keys[NT * IT];
    uint32_t vals[NT * IT];
};

// One stable counting pass of the block over digit bits [lo, lo + width):
// rows move (through shared memory) from their current sequence position to
// their place in digit order.  Returns false when every row has the same digit
// (nothing moves).  Leaves the digit counts in sm.cnt and the exclusive digit
// offsets in sm.doff.  `to_smem_only`: rows stay in shared memory (the caller
// reads them there) instead of being reloaded into registers.
template <typename K, int NT, int IT, int RANK>
__device__ __forceinline__ bool block_pass(BlockSmem<K, NT, IT> &sm, K (&key)[IT], uint32_t (&val)[IT],
                                           uint32_t steps, uint32_t wbase, uint32_t len, uint32_t lo,
                                           uint32_t width, bool to_smem_only)
{
    constexpr int NW = NT / 32;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (int d = lane; d < kRadix; d += 32) sm.whist[warp][d] = 0;
    if (threadIdx.x == 0) {
        sm.flag = 0;
        sm.maxb = 0;
    }
    __syncthreads();
    uint32_t rank[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        if (j < (int)steps) {   // uniform across the block
            const uint32_t p = wbase + j * 32 + lane;
            rank[j] = wlms_rank<RANK>(digit_of(key[j], lo, width), p < len, sm.whist[warp], width);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += NT) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const uint32_t c = sm.whist[w][d];
            sm.whist[w][d] = run;
            run += c;
        }
        sm.doff[d] = run;
        sm.cnt[d] = run;
        if (run == len) sm.flag = 1;   // one digit holds every row: identity pass
        if (run) atomicMax(&sm.maxb, run);
    }
    __syncthreads();
    const bool identity = sm.flag != 0;
    __syncthreads();
    if (identity) return false;   // uniform across the block
    uint32_t tot;
    block_exclusive_scan_radix<NT>(sm.doff, sm.tmp, &tot);
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t p = wbase + j * 32 + lane;
        if (j < (int)steps && p < len) {
            const uint32_t d = digit_of(key[j], lo, width);
            const uint32_t pos = sm.doff[d] + sm.whist[warp][d] + rank[j];
            sm.keys[pos] = key[j];
            sm.vals[pos] = val[j];
        }
    }
    __syncthreads();
    if (!to_smem_only) {
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            if (j < (int)steps && p < len) { key[j] = sm.keys[p]; val[j] = sm.vals[p]; }
        }
        __syncthreads();
    }
    return true;
}

// The stable fallback of the block sort (see above) for one segment; rows
// are loaded again from HBM.  Kept out of line so that its register demand
// does not weigh on the fast path.
template <typename K, int NT, int IT, int RANK>
__device__ __noinline__ void block_sort_fallback(BlockSmem<K, NT, IT> &sm, Bufs<K> b, uint32_t start, uint32_t len,
                                                 uint32_t shift, uint32_t src)
{
    constexpr int NW = NT / 32;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t steps = (len + NW * 32 - 1) / (NW * 32);
    const uint32_t wbase = warp * steps * 32;
    K key[IT];
    uint32_t val[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
        const uint32_t p = wbase + j * 32 + lane;
        key[j] = 0;
        val[j] = 0;
        if (j < (int)steps && p < len) load_kv(b, src, (uint64_t)start + p, key[j], val[j]);
    }
    bool written = false;
    uint32_t lsd_top = shift;   // LSD passes cover [0, lsd_top)
    if (shift > (uint32_t)kRadixBits) {
        const uint32_t top = shift - kRadixBits;
        const bool moved = block_pass<K, NT, IT, RANK>(sm, key, val, steps, wbase, len, top, kRadixBits, true);
        if (!moved) {
            lsd_top = top;   // the top digit is constant: sort the bits below it
        } else if (sm.maxb <= kCountRankMax) {
            // rows are in smem in top-digit order; rank each row inside its bucket
            for (uint32_t p = threadIdx.x; p < len; p += NT) {
                const K k = sm.keys[p];
                const uint32_t v = sm.vals[p];
                const uint32_t d = digit_of(k, top, kRadixBits);
                const uint32_t b0 = sm.doff[d];
                const uint32_t b1 = b0 + sm.cnt[d];
                uint32_t r = 0;
                for (uint32_t q = b0; q < b1; ++q) {
                    const K kq = sm.keys[q];
                    r += (kq < k) || (kq == k && q < p);
                }
                b.k0[(uint64_t)start + b0 + r] = k;
                b.v0[(uint64_t)start + b0 + r] = v;
            }
            written = true;
        } else {
            // skewed: continue from the split order with LSD passes below the
            // top digit, then the top digit again
#pragma unroll
            for (int j = 0; j < IT; ++j) {
                const uint32_t p = wbase + j * 32 + lane;
                if (j < (int)steps && p < len) { key[j] = sm.keys[p]; val[j] = sm.vals[p]; }
            }
            __syncthreads();
            for (uint32_t lo = 0; lo < top; lo += kRadixBits)
                block_pass<K, NT, IT, RANK>(sm, key, val, steps, wbase, len, lo, min((uint32_t)kRadixBits, top - lo),
                                            false);
            block_pass<K, NT, IT, RANK>(sm, key, val, steps, wbase, len, top, kRadixBits, false);
            lsd_top = 0;
        }
    }
    if (!written) {
        for (uint32_t lo = 0; lo < lsd_top; lo += kRadixBits)
            block_pass<K, NT, IT, RANK>(sm, key, val, steps, wbase, len, lo, min((uint32_t)kRadixBits, lsd_top - lo),
                                        false);
        // every load of this segment is done (barriers above) before the
        // first store into BUF0, which may alias the EXT oids of the range
        __syncthreads();
#pragma unroll
        for (int j = 0; j < IT; ++j) {
            const uint32_t p = wbase + j * 32 + lane;
            if (j < (int)steps && p < len) {
                b.k0[(uint64_t)start + p] = key[j];
                b.v0[(uint64_t)start + p] = val[j];
            }
        }
    }
}

// 1024 threads per SM for every tier (64 registers a thread).
template <typename K, int NT, int IT, int RANK>
__global__ void __launch_bounds__(NT, 1024 / NT)
block_sort_kernel(Bufs<K> b, const uint2 *list, const uint32_t *d_count)
{
    kernel_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = NT / 32;
    const uint32_t count = *d_count;
    const int warp = threadIdx.x >> 5;
    for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
        const uint2 ent = list[e];
        const uint32_t start = ent.x;
        const uint32_t len = ent.y & 0xFFFFu;
        const uint32_t shift = (ent.y >> 16) & 0x7Fu;
        const uint32_t src = (ent.y >> 24) & 3u;
        // Spread the segment evenly over the warps: warp w owns positions
        // [w*steps*32, (w+1)*steps*32); a step is one item per lane.
        const uint32_t steps = (len + NW * 32 - 1) / (NW * 32);
        const uint32_t wbase = warp * steps * 32;
        K key[IT];
        uint32_t val[IT];
        load_rows<K, IT>(b, src, start, len, steps, wbase, key, val);
        if (!bucket_rank_sort<K, NT, IT>(*reinterpret_cast<BucketSmem<K, NT, IT> *>(smem_raw), key, val, steps, wbase,
                                         len, b, start)) {
            block_sort_fallback<K, NT, IT, RANK>(*reinterpret_cast<BlockSmem<K, NT, IT> *>(smem_raw), b, start, len,
                                                 shift, src);
            __syncthreads();
        }
    }
}

// Thread-per-segment sort of tiny segments (2..kCapT rows): the rows sit in
// registers and an odd-even transposition network of N rounds sorts them.
// It swaps only strictly inverted neighbours, so equal keys keep their order
// (stable); the padding slots hold the largest key and stay behind the rows.
template <typename K, int N>
__device__ __forceinline__ void sort_tiny(const Bufs<K> &b, uint32_t start, uint32_t len, uint32_t src)
{
    K k[N];
    uint32_t v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        k[i] = ~K(0);
        v[i] = 0;
        if (i < (int)len) load_kv(b, src, (uint64_t)start + i, k[i], v[i]);
    }
#pragma unroll
    for (int r = 0; r < N; ++r) {
#pragma unroll
        for (int i = r & 1; i + 1 < N; i += 2) {
            if (k[i] > k[i + 1]) {
                const K tk = k[i];
                k[i] = k[i + 1];
                k[i + 1] = tk;
                const uint32_t tv = v[i];
                v[i] = v[i + 1];
                v[i + 1] = tv;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (i < (int)len) {
            b.k0[(uint64_t)start + i] = k[i];
            b.v0[(uint64_t)start + i] = v[i];
        }
    }
}

template <typename K, int NMAX>
__global__ void __launch_bounds__(256) thread_sort_kernel(Bufs<K> b, const uint2 *list, const uint32_t *d_count)
{
    kernel_prologue();
    const uint32_t count = *d_count;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const uint2 ent = list[e];
        const uint32_t start = ent.x;
        const uint32_t len = ent.y & 0xFFFFu;
        const uint32_t src = (ent.y >> 24) & 3u;
        if constexpr (NMAX > 16) {
            sort_tiny<K, NMAX>(b, start, len, src);
        } else {
            if (len <= 2) sort_tiny<K, 2>(b, start, len, src);
            else if (len <= 4) sort_tiny<K, 4>(b, start, len, src);
            else if (len <= 8) sort_tiny<K, 8>(b, start, len, src);
            else sort_tiny<K, 16>(b, start, len, src);
        }
    }
}

// Warp-per-segment LSD radix sort (len <= 32 * kItemsA), stable.
template <typename K>
struct WarpSmem {
    uint32_t hist[kRadix];
    K keys[32 * kItemsA];
    uint32_t vals[32 * kItemsA];
};

template <typename K, int RANK>
__global__ void __launch_bounds__(256) warp_sort_kernel(Bufs<K> b, const uint2 *list, const uint32_t *d_count)
{
    kernel_prologue();
    __shared__ WarpSmem<K> all[8];
    WarpSmem<K> &sm = all[threadIdx.x >> 5];
    const uint32_t count = *d_count;
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * 8;
    for (uint32_t e = blockIdx.x * 8 + (threadIdx.x >> 5); e < count; e += nwarps) {
        const uint2 ent = list[e];
        const uint32_t start = ent.x;
        const uint32_t len = ent.y & 0xFFFFu;
        const uint32_t shift = (ent.y >> 16) & 0x7Fu;
        const uint32_t src = (ent.y >> 24) & 3u;
        K key[kItemsA];
        uint32_t val[kItemsA];
#pragma unroll
        for (int j = 0; j < kItemsA; ++j) {
            const uint32_t p = j * 32 + lane;
            if (p < len) load_kv(b, src, (uint64_t)start + p, key[j], val[j]);
            else { key[j] = 0; val[j] = 0; }
        }
        for (uint32_t lo = 0; lo < shift; lo += kRadixBits) {
            const uint32_t width = min((uint32_t)kRadixBits, shift - lo);
#pragma unroll
            for (int d = lane; d < kRadix; d += 32) sm.hist[d] = 0;
            __syncwarp();
            uint32_t rank[kItemsA];
            uint32_t dig[kItemsA];
#pragma unroll
            for (int j = 0; j < kItemsA; ++j) {
                const uint32_t p = j * 32 + lane;
                dig[j] = digit_of(key[j], lo, width);
                rank[j] = wlms_rank<RANK>(dig[j], p < len, sm.hist, width);
            }
            // warp exclusive scan of the 256 counters (8 per lane)
            uint32_t c[8];
            uint32_t sum = 0;
            bool full = false;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                c[i] = sm.hist[lane * 8 + i];
                full |= (c[i] == len);
                sum += c[i];
            }
            if (__any_sync(0xFFFFFFFFu, full)) continue;   // identity pass
            uint32_t incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += y;
            }
            uint32_t run = incl - sum;
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                sm.hist[lane * 8 + i] = run;
                run += c[i];
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < kItemsA; ++j) {
                const uint32_t p = j * 32 + lane;
                if (p < len) {
                    const uint32_t pos = sm.hist[dig[j]] + rank[j];
                    sm.keys[pos] = key[j];
                    sm.vals[pos] = val[j];
                }
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < kItemsA; ++j) {
                const uint32_t p = j * 32 + lane;
                if (p < len) { key[j] = sm.keys[p]; val[j] = sm.vals[p]; }
            }
            __syncwarp();
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < kItemsA; ++j) {
            const uint32_t p = j * 32 + lane;
            if (p < len) {
                b.k0[(uint64_t)start + p] = key[j];
                b.v0[(uint64_t)start + p] = val[j];
            }
        }
        __syncwarp();
    }
}

// Segments that need no sorting but sit outside BUF0: one warp per entry.
template <typename K>
__global__ void __launch_bounds__(256) copy_kernel(Bufs<K> b, const LargeSeg *list, const uint32_t *d_count)
{
    kernel_prologue();
    const uint32_t count = *d_count;
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * (blockDim.x / 32);
    for (uint32_t e = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); e < count; e += nwarps) {
        const LargeSeg sg = list[e];
        for (uint32_t i = lane; i < sg.len; i += 32) {
            const uint64_t r = (uint64_t)sg.start + i;
            K k;
            uint32_t v;
            load_kv(b, sg.src & 3u, r, k, v);
            b.k0[r] = k;
            b.v0[r] = v;
        }
    }
}

// Large segments that only need to reach BUF0: tiles of kCopySplit rows
// spread over the whole grid (tile -> segment by binary search).
template <typename K>
__global__ void __launch_bounds__(256) copy_tiles_kernel(Bufs<K> b, const LargeSeg *list, const uint32_t *d_count,
                                                         const uint32_t *tile_prefix)
{
    kernel_prologue();
    const uint32_t count = *d_count;
    if (count == 0) return;
    const uint32_t T = tile_prefix[count];
    for (uint32_t t = blockIdx.x; t < T; t += gridDim.x) {
        const uint32_t s = find_segment_warp(tile_prefix, count, t);
        const LargeSeg sg = list[s];
        const uint64_t beg = (uint64_t)sg.start + (uint64_t)(t - tile_prefix[s]) * kCopySplit;
        const uint64_t end = min((uint64_t)sg.start + sg.len, beg + kCopySplit);
        for (uint64_t r = beg + threadIdx.x; r < end; r += blockDim.x) {
            K k;
            uint32_t v;
            load_kv(b, sg.src & 3u, r, k, v);
            b.k0[r] = k;
            b.v0[r] = v;
        }
    }
}

template <typename F>
int set_smem(fmcs_ctx *ctx, F *f, size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "cudaFuncSetAttribute");
}

#define FMCS_LAUNCH_CHECK(what)                                         \
    do {                                                                \
        cudaError_t e_ = cudaGetLastError();                            \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what);          \
    } while (0)

template <typename K, int RANK, int IT>
int sort_segments_t(fmcs_ctx *ctx, const SortArgs &a)
{
    const uint64_t n = a.n;
    cudaStream_t st = ctx->stream;
    // buffers
    Bufs<K> b;
    b.ext_bank = (const K *)a.bank;
    b.ext_order = a.order_in;
    void *p = nullptr;
    int rc;
    if (a.keys_out) {
        b.k0 = (K *)a.keys_out;
    } else {
        if ((rc = ws_get(ctx, kSlotKeys0, n * sizeof(K), &p))) return rc;
        b.k0 = (K *)p;
    }
    b.v0 = a.order_out;
    if ((rc = ws_get(ctx, kSlotKeys1, n * sizeof(K), &p))) return rc;
    b.k1 = (K *)p;
    if ((rc = ws_get(ctx, kSlotVals1, n * sizeof(uint32_t), &p))) return rc;
    b.v1 = (uint32_t *)p;

    // lists (capacities are bounds on disjoint segments of each tier's minimum size)
    const uint32_t local_max = std::max<uint32_t>(kCapA, std::min<uint32_t>(ctx->local_max, kCapLocal));
    const uint32_t tile_rows = kNtM * IT;
    const uint64_t cap_large = n / (local_max + 1) + 2;
    const uint64_t cap_t = n / 2 + 2, cap_t32 = n / (kCapT + 1) + 2, cap_a = n / (kCapT + 1) + 2;
    const uint64_t cap_b1 = n / (kCapA + 1) + 2;
    const uint64_t cap_b2 = n / (kCapB1 + 1) + 2;
    const uint64_t cap_c1 = n / (kCapB2 + 1) + 2, cap_c1b = n / (kCapC1 + 1) + 2, cap_c2 = n / (kCapC1b + 1) + 2;
    const uint64_t cap_c3 = n / (kCapC2 + 1) + 2;
    // copy entries: disjoint ranges; at most 256 children per large segment per
    // level, so bounded by both n and (levels + 1) * 256 * cap_large
    const uint64_t levels_max = (a.key_bits + kRadixBits - 1) / kRadixBits;
    const uint64_t cap_copy = std::min<uint64_t>(n, (levels_max + 1) * kRadix * cap_large) + 2;
    LargeSeg *large[2];
    if ((rc = ws_get(ctx, kSlotLarge0, cap_large * sizeof(LargeSeg), &p))) return rc;
    large[0] = (LargeSeg *)p;
    if ((rc = ws_get(ctx, kSlotLarge1, cap_large * sizeof(LargeSeg), &p))) return rc;
    large[1] = (LargeSeg *)p;
    Lists lists;
    {
        const size_t e = sizeof(uint2);
        if ((rc = ws_get(ctx, kSlotLocalA,
                         carve_total({cap_t * e, cap_t32 * e, cap_a * e, cap_b1 * e, cap_b2 * e, cap_c1 * e,
                                      cap_c1b * e, cap_c2 * e, cap_c3 * e}),
                         &p)))
            return rc;
        Carver cv(p);
        lists.t = cv.take<uint2>(cap_t);
        lists.t32 = cv.take<uint2>(cap_t32);
        lists.a = cv.take<uint2>(cap_a);
        lists.cap_t32 = sizeof(K) <= 4 ? kCapT32 : 0;
        lists.b1 = cv.take<uint2>(cap_b1);
        lists.b2 = cv.take<uint2>(cap_b2);
        lists.c1 = cv.take<uint2>(cap_c1);
        lists.c1b = cv.take<uint2>(cap_c1b);
        lists.c2 = cv.take<uint2>(cap_c2);
        lists.c3 = cv.take<uint2>(cap_c3);
        if ((rc = ws_get(ctx, kSlotLocalC, carve_total({cap_copy * sizeof(LargeSeg), cap_large * sizeof(LargeSeg)}),
                         &p)))
            return rc;
        Carver cc(p);
        lists.copy = cc.take<LargeSeg>(cap_copy);
        lists.copy_large = cc.take<LargeSeg>(cap_large);
        lists.local_max = local_max;
    }
    // histogram rows: one per chunk of kChunkTiles tiles of a large segment
    // (a segment's chunks <= its tiles / kChunkTiles + 1)
    const uint64_t max_tiles = n / tile_rows + cap_large + 1;
    const uint64_t cap_chunks = max_tiles / kChunkTiles + cap_large + 1;
    uint32_t *hists[2], *tile_prefix, *chunk_prefix;
    if ((rc = ws_get(ctx, kSlotSegHist, 2 * carve_round(cap_chunks * kRadix * sizeof(uint32_t)), &p))) return rc;
    {
        Carver cv(p);
        hists[0] = cv.take<uint32_t>(cap_chunks * kRadix);
        hists[1] = cv.take<uint32_t>(cap_chunks * kRadix);
    }
    if ((rc = ws_get(ctx, kSlotTilePrefix, carve_total({(cap_large + 1) * sizeof(uint32_t),
                                                        (cap_large + 1) * sizeof(uint32_t)}), &p)))
        return rc;
    {
        Carver cv(p);
        tile_prefix = cv.take<uint32_t>(cap_large + 1);
        chunk_prefix = cv.take<uint32_t>(cap_large + 1);
    }
    unsigned long long *lookback;
    if ((rc = ws_get(ctx, kSlotLookback, max_tiles * kRadix * sizeof(unsigned long long), &p, true))) return rc;
    lookback = (unsigned long long *)p;
    uint32_t *ctr;
    if ((rc = ws_get(ctx, kSlotCounters, 4096, &p))) return rc;
    ctr = (uint32_t *)p + 64;   // words 0..63 belong to other kernels
    cudaMemsetAsync(ctr, 0, kCtrWords * sizeof(uint32_t), st);

    const int sms = ctx->num_sms;
    // classification of the initial segments
    {
        const uint32_t *seg_start = a.seg_start;
        const uint32_t *d_nseg = a.d_nseg;
        unsigned grid = seg_start ? (unsigned)std::min<uint64_t>((a.nseg_host + 255) / 256 + 1, (uint64_t)sms * 16)
                                  : 1u;
        if (seg_start && a.nseg_host == 0) grid = (unsigned)sms * 16;
        { LaunchScope ls_(ctx, "classify");
            launch_k(classify_kernel<K>, grid, 256, 0, st, b, seg_start, d_nseg, n, a.key_bits, ctr, large[0], lists,
                     seg_start ? nullptr : a.top_hist, a.d_key_bits, a.d_in_order);
        }
        FMCS_LAUNCH_CHECK("classify");
    }
    // The host's copy of the counters (ctx->h_small + 16) when an eager call
    // has read them back after the last routing of segments to the tiers.
    bool tiers_known = false;
    const uint32_t *hctr = ctx->h_small + 16;
    if (!a.fixed_launches && !a.seg_start && !a.d_key_bits && !a.d_in_order && n <= (uint64_t)local_max) {
        // round 0 that fits one tier: the host routes it as classify does
        uint32_t *w = ctx->h_small + 16;
        for (int i = 0; i < kCtrWords; ++i) w[i] = 0;
        const uint32_t len = (uint32_t)n;
        if (len > 1) {
            const int which = len <= (uint32_t)kCapT ? kCtrLocalT
                              : len <= lists.cap_t32 ? kCtrLocalT32
                              : len <= (uint32_t)kCapA ? kCtrLocalA
                              : len <= (uint32_t)kCapB1 ? kCtrLocalB1
                              : len <= (uint32_t)kCapB2 ? kCtrLocalB2
                              : len <= (uint32_t)kCapC1 ? kCtrLocalC1
                              : len <= (uint32_t)kCapC1b ? kCtrLocalC1b
                              : len <= (uint32_t)kCapC2 ? kCtrLocalC2 : kCtrLocalC3;
            w[which] = 1;
        }
        tiers_known = true;
    }
    // MSD levels
    const int levels = (int)((a.key_bits + kRadixBits - 1) / kRadixBits);
    const size_t msd_smem = sizeof(MsdSmem<K, IT>);
    if ((rc = set_smem(ctx, msd_scatter_kernel<K, RANK, IT>, msd_smem))) return rc;
    if (n > (uint64_t)local_max) {
        // Host-known count of the level's large segments (exact unless the
        // caller asked for a fixed launch sequence, e.g. for graph capture).
        uint32_t nlarge = 1;
        if (a.fixed_launches) {
            nlarge = 1;
        } else if (a.seg_start) {
            cudaMemcpyAsync(ctx->h_small + 16, ctr, kCtrWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "sort: level count");
            nlarge = ctx->h_small[16 + kCtrLarge0];
            tiers_known = true;
        }
        const int hist0_ready = (a.top_hist && !a.seg_start) ? 1 : 0;
        const LevelRefs lr{{large[0], large[1]}, {hists[0], hists[1]}, ctr, 1, hist0_ready, chunk_prefix,
                           hist0_ready ? a.top_hist : nullptr};
        const uint32_t epoch_base = ctx->epoch;
        ctx->epoch += (uint32_t)levels;
        const unsigned scatter_grid = sms * msd_ctas_per_sm(IT);
        int host_lvl = 0;   // the level being launched, for the eager read-back
        // one level: the same four launches for every level (the level index
        // lives on the device)
        auto level = [&](cudaStream_t s, cudaGraphConditionalHandle more, bool read_back) -> int {
            { LaunchScope ls_(ctx, "tile_prefix");
                launch_k(level_prefix_kernel, 1, 1024, 0, s, lr, tile_prefix, tile_rows);
            }
            if (!(hist0_ready && host_lvl == 0 && read_back)) {
                // (inside a graph the launch stays and returns at once on level 0)
                LaunchScope ls_(ctx, "msd_hist");
                launch_k(msd_hist_kernel<K>, sms * kHistCtas, kNtM, 0, s, b, lr, tile_prefix, tile_rows);
            }
            { LaunchScope ls_(ctx, "msd_plan");
                launch_k(msd_plan_kernel, sms * 8, kPlanThreads, 0, s, lr, lists, true, tile_rows);
            }
            if (read_back) {
                // read the counters (the next level's count, the rows moved,
                // the tiers' list sizes) while the scatter runs
                cudaMemcpyAsync(ctx->h_small + 16, ctr, kCtrWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
                cudaEventRecord(ctx->ev_level, s);
            }
            {
                LaunchScope ls_(ctx, "msd_scatter");
                launch_k(msd_scatter_kernel<K, RANK, IT>, scatter_grid, kNtM, msd_smem, s, b, lr, tile_prefix, lookback,
                                                                                   epoch_base, ctx->d_status, more,
                                                                                   (uint32_t)levels);
                if (read_back) {
                    cudaError_t e = cudaEventSynchronize(ctx->ev_level);
                    if (e != cudaSuccess) return cuda_fail(ctx, e, "sort: level event");
                    // algorithmic bytes: every moved row is read from the level's
                    // source (the round's bank, through the order when there is
                    // one, at level 0; the work buffers after) and written once
                    const double moved = (double)ctx->h_small[16 + kCtrMoved];
                    const double rd = host_lvl == 0 ? (double)sizeof(K) + (b.ext_order ? 4.0 : 0.0)
                                                    : (double)sizeof(K) + 4.0;
                    ls_.set_units(moved);
                    ls_.set_bytes(moved * (rd + (double)sizeof(K) + 4.0));
                }
            }
            FMCS_LAUNCH_CHECK("msd level");
            return FMCS_OK;
        };
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (a.fixed_launches && cudaStreamIsCapturing(st, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusActive) {
            // graph capture: the levels are one WHILE node whose body is one
            // level; each level's scatter decides whether another follows
            if ((rc = capture_while(ctx, st, [&](cudaStream_t s, cudaGraphConditionalHandle h) {
                     return level(s, h, false);
                 })))
                return rc;
        } else {
            for (int lvl = 0; lvl < levels && nlarge > 0; ++lvl) {
                host_lvl = lvl;
                if ((rc = level(st, 0, !a.fixed_launches))) return rc;
                if (!a.fixed_launches) {
                    nlarge = ctx->h_small[16 + kCtrLarge0 + ((uint32_t)(lvl + 1) & 1u)];
                    tiers_known = true;
                }
            }
        }
    }
    // local tiers
    const size_t smem_b1 = std::max(sizeof(BlockSmem<K, kNtB1, kItB1>), sizeof(BucketSmem<K, kNtB1, kItB1>));
    const size_t smem_b2 = std::max(sizeof(BlockSmem<K, kNtB2, kItB2>), sizeof(BucketSmem<K, kNtB2, kItB2>));
    const size_t smem_c1 = std::max(sizeof(BlockSmem<K, kNtC1, kItC1>), sizeof(BucketSmem<K, kNtC1, kItC1>));
    const size_t smem_c1b = std::max(sizeof(BlockSmem<K, kNtC1b, kItC1b>), sizeof(BucketSmem<K, kNtC1b, kItC1b>));
    const size_t smem_c2 = std::max(sizeof(BlockSmem<K, kNtC2, kItC2>), sizeof(BucketSmem<K, kNtC2, kItC2>));
    const size_t smem_c3 = std::max(sizeof(BlockSmem<K, kNtC3, kItC3>), sizeof(BucketSmem<K, kNtC3, kItC3>));
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtB1, kItB1, RANK>, smem_b1))) return rc;
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtB2, kItB2, RANK>, smem_b2))) return rc;
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtC1, kItC1, RANK>, smem_c1))) return rc;
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtC1b, kItC1b, RANK>, smem_c1b))) return rc;
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtC2, kItC2, RANK>, smem_c2))) return rc;
    if ((rc = set_smem(ctx, block_sort_kernel<K, kNtC3, kItC3, RANK>, smem_c3))) return rc;
    // Each tier's launch, with the counter word of its list.  An eager call
    // that knows the lists' sizes from its last read-back (tiers_known) does
    // not launch a tier whose list is empty.  A captured graph launches every
    // tier (an empty one returns at once): one conditional node per tier cost
    // more on replay than the empty launches it saved.
    struct Tier {
        int word;
        std::function<void(cudaStream_t)> launch;
    };
    std::vector<Tier> tiers;
    tiers.push_back({kCtrLocalT, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "thread_sort");
        launch_k(thread_sort_kernel<K, 16>, sms * 8, 256, 0, s, b, lists.t, &ctr[kCtrLocalT]);
    }});
    if constexpr (sizeof(K) <= 4) {
        tiers.push_back({kCtrLocalT32, [&](cudaStream_t s) {
            LaunchScope ls_(ctx, "thread_sort_32");
            launch_k(thread_sort_kernel<K, 32>, sms * 8, 256, 0, s, b, lists.t32, &ctr[kCtrLocalT32]);
        }});
    }
    tiers.push_back({kCtrLocalA, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "warp_sort");
        launch_k(warp_sort_kernel<K, RANK>, sms * 16, 256, 0, s, b, lists.a, &ctr[kCtrLocalA]);
    }});
    tiers.push_back({kCtrLocalB1, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_512");
        launch_k(block_sort_kernel<K, kNtB1, kItB1, RANK>, sms * (1024 / kNtB1), kNtB1, smem_b1, s, b, lists.b1,
                 &ctr[kCtrLocalB1]);
    }});
    tiers.push_back({kCtrLocalB2, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_1024");
        launch_k(block_sort_kernel<K, kNtB2, kItB2, RANK>, sms * (1024 / kNtB2), kNtB2, smem_b2, s, b, lists.b2,
                 &ctr[kCtrLocalB2]);
    }});
    tiers.push_back({kCtrLocalC1, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_2048");
        launch_k(block_sort_kernel<K, kNtC1, kItC1, RANK>, sms * (1024 / kNtC1), kNtC1, smem_c1, s, b, lists.c1,
                 &ctr[kCtrLocalC1]);
    }});
    tiers.push_back({kCtrLocalC1b, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_2304");
        launch_k(block_sort_kernel<K, kNtC1b, kItC1b, RANK>, sms * (1024 / kNtC1b), kNtC1b, smem_c1b, s, b, lists.c1b,
                 &ctr[kCtrLocalC1b]);
    }});
    tiers.push_back({kCtrLocalC2, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_4096");
        launch_k(block_sort_kernel<K, kNtC2, kItC2, RANK>, sms * (1024 / kNtC2), kNtC2, smem_c2, s, b, lists.c2,
                 &ctr[kCtrLocalC2]);
    }});
    tiers.push_back({kCtrLocalC3, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "block_sort_8192");
        launch_k(block_sort_kernel<K, kNtC3, kItC3, RANK>, sms * (1024 / kNtC3), kNtC3, smem_c3, s, b, lists.c3,
                 &ctr[kCtrLocalC3]);
    }});
    tiers.push_back({kCtrCopy, [&](cudaStream_t s) {
        LaunchScope ls_(ctx, "copy");
        launch_k(copy_kernel<K>, sms * 4, 256, 0, s, b, lists.copy, &ctr[kCtrCopy]);
    }});
    tiers.push_back({kCtrCopyLarge, [&](cudaStream_t s) {
        {
            LaunchScope ls_(ctx, "tile_prefix");
            launch_k(tile_prefix_kernel, 1, 1024, 0, s, lists.copy_large, &ctr[kCtrCopyLarge], tile_prefix,
                     &ctr[kCtrCopyTile], kCopySplit);
        }
        LaunchScope ls_(ctx, "copy_tiles");
        launch_k(copy_tiles_kernel<K>, sms * 8, 256, 0, s, b, lists.copy_large, &ctr[kCtrCopyLarge], tile_prefix);
    }});
    // The tiers' segments are disjoint: the tiers up to the 2048-row one run
    // on the context's stream, the larger ones and the copies on its second
    // stream at the same time, so that a tier with few segments (one wave of
    // one segment per CTA, latency-bound) overlaps a busy one.  While
    // profiling, every tier stays on the context's stream (one at a time,
    // each timed alone).
    auto wanted = [&](const Tier &t) { return !tiers_known || hctr[t.word] > 0; };
    size_t split = 0;
    while (split < tiers.size() && tiers[split].word != kCtrLocalC1b) ++split;
    bool two = !ctx->prof_on;
    if (two) {
        bool a = false, bb = false;
        for (size_t i = 0; i < tiers.size(); ++i) (i < split ? a : bb) |= wanted(tiers[i]);
        two = a && bb;
    }
    if (two) {
        if ((rc = fork_par(ctx, st))) return rc;
        for (size_t i = 0; i < tiers.size(); ++i)
            if (wanted(tiers[i])) tiers[i].launch(i < split ? st : ctx->par);
        if ((rc = join_par(ctx, st))) return rc;
    } else {
        for (const Tier &t : tiers)
            if (wanted(t)) t.launch(st);
    }
    FMCS_LAUNCH_CHECK("local tiers");
    return FMCS_OK;
}

// ---------------------------------------------------------------------------
// Full-array LSD radix sort (the plain comparator path: no segments, no
// binning).  One pass per 8 key bits, each pass the MSD level kernels applied
// to a single segment [0, n) with the digit at bits [shift-8, shift).  Passes
// where every row has the same digit are skipped on the device, so the buffer
// holding the result is tracked on the device and a final copy puts it in
// BUF0.
// ---------------------------------------------------------------------------
__global__ void lsd_set_pass_kernel(LargeSeg *seg, uint32_t *hist_row, uint32_t *nseg, uint32_t n, uint32_t shift,
                                    int first)
{
    kernel_prologue();
    if (threadIdx.x == 0) {
        uint32_t src = kSrcBuf0;
        if (!first) {
            const LargeSeg prev = seg[0];
            src = (prev.src & kSkipBit) ? (prev.src & 3u) : ((prev.src & 3u) == kSrcBuf1 ? kSrcBuf0 : kSrcBuf1);
        }
        seg[0] = LargeSeg{0, n, shift, src};
        *nseg = 1;
    }
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist_row[d] = 0;
}

template <typename K>
__global__ void lsd_finalize_kernel(Bufs<K> b, const LargeSeg *seg, uint64_t n)
{
    kernel_prologue();
    const LargeSeg last = seg[0];
    const uint32_t where = (last.src & kSkipBit) ? (last.src & 3u) : ((last.src & 3u) == kSrcBuf1 ? kSrcBuf0 : kSrcBuf1);
    if (where != kSrcBuf1) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        b.k0[i] = b.k1[i];
        b.v0[i] = b.v1[i];
    }
}

template <typename K, int RANK, int IT>
int lsd_sort_full_t(fmcs_ctx *ctx, void *keys, uint32_t *vals, uint64_t n, uint32_t bits)
{
    cudaStream_t st = ctx->stream;
    int rc;
    void *p;
    Bufs<K> b;
    b.k0 = (K *)keys;
    b.v0 = vals;
    b.ext_bank = nullptr;
    b.ext_order = nullptr;
    if ((rc = ws_get(ctx, kSlotKeys1, n * sizeof(K), &p))) return rc;
    b.k1 = (K *)p;
    if ((rc = ws_get(ctx, kSlotVals1, n * sizeof(uint32_t), &p))) return rc;
    b.v1 = (uint32_t *)p;
    LargeSeg *seg;
    if ((rc = ws_get(ctx, kSlotLarge0, sizeof(LargeSeg) * 2, &p))) return rc;
    seg = (LargeSeg *)p;
    uint32_t *hist, *tile_prefix;
    if ((rc = ws_get(ctx, kSlotSegHist, 2 * kRadix * sizeof(uint32_t), &p))) return rc;
    hist = (uint32_t *)p;
    if ((rc = ws_get(ctx, kSlotTilePrefix, 4 * sizeof(uint32_t), &p))) return rc;
    tile_prefix = (uint32_t *)p;
    const uint32_t tile_rows = kNtM * IT;
    const uint64_t max_tiles = n / tile_rows + 2;
    unsigned long long *lookback;
    if ((rc = ws_get(ctx, kSlotLookback, max_tiles * kRadix * sizeof(unsigned long long), &p, true))) return rc;
    lookback = (unsigned long long *)p;
    uint32_t *ctr;
    if ((rc = ws_get(ctx, kSlotCounters, 4096, &p))) return rc;
    ctr = (uint32_t *)p + 64;
    const size_t msd_smem = sizeof(MsdSmem<K, IT>);
    if ((rc = set_smem(ctx, msd_scatter_kernel<K, RANK, IT>, msd_smem))) return rc;
    const int sms = ctx->num_sms;
    Lists none{};
    // one segment [0, n), re-set before every pass; level buffers of set 0
    const LevelRefs lr{{seg, seg + 1}, {hist, hist + kRadix}, ctr, 0, 0};
    int pass = 0;
    for (uint32_t lo = 0; lo < bits; lo += kRadixBits, ++pass) {
        const uint32_t shift = std::min(bits, lo + kRadixBits);
        { LaunchScope ls_(ctx, "lsd_set_pass");
            launch_k(lsd_set_pass_kernel, 1, 256, 0, st, seg, hist, &ctr[kCtrLarge0], (uint32_t)n, shift, pass == 0);
        }
        { LaunchScope ls_(ctx, "tile_prefix");
            launch_k(level_prefix_kernel, 1, 1024, 0, st, lr, tile_prefix, tile_rows);
        }
        { LaunchScope ls_(ctx, "msd_hist");
            launch_k(msd_hist_kernel<K>, sms * kHistCtas, kNtM, 0, st, b, lr, tile_prefix, tile_rows);
        }
        { LaunchScope ls_(ctx, "msd_plan");
            launch_k(msd_plan_kernel, 1, kPlanThreads, 0, st, lr, none, false, tile_rows);
        }
        { LaunchScope ls_(ctx, "msd_scatter");
            launch_k(msd_scatter_kernel<K, RANK, IT>, sms * msd_ctas_per_sm(IT), kNtM, msd_smem, st, 
                b, lr, tile_prefix, lookback, ctx->epoch++, ctx->d_status, 0, 1u);
        }
        FMCS_LAUNCH_CHECK("lsd pass");
    }
    if (pass > 0) {
        LaunchScope ls_(ctx, "lsd_finalize");
        launch_k(lsd_finalize_kernel<K>, sms * 8, 256, 0, st, b, seg, n);
    }
    FMCS_LAUNCH_CHECK("lsd finalize");
    return FMCS_OK;
}

}  // namespace

uint32_t msd_chunk_rows(const fmcs_ctx *ctx)
{
    return kChunkTiles * (uint32_t)kNtM * (ctx->msd_items >= 16 ? 16u : 8u);
}

int lsd_sort_full(fmcs_ctx *ctx, void *keys, uint32_t key_bytes, uint32_t *vals, uint64_t n, uint32_t bits)
{
    if (n <= 1 || bits == 0) return FMCS_OK;
    switch (key_bytes) {
    case 4: return lsd_sort_full_t<uint32_t, kRankMatch, 8>(ctx, keys, vals, n, bits);
    case 8: return lsd_sort_full_t<uint64_t, kRankMatch, 8>(ctx, keys, vals, n, bits);
    case 2: return lsd_sort_full_t<uint16_t, kRankMatch, 8>(ctx, keys, vals, n, bits);
    default: return set_error(ctx, FMCS_E_INVAL, "lsd sort: key bytes must be 2, 4 or 8");
    }
}

template <typename K>
static int sort_dispatch(fmcs_ctx *ctx, const SortArgs &a)
{
    const bool big = ctx->msd_items >= 16;
    if (ctx->rank_mode == 2)
        return big ? sort_segments_t<K, kRankOr, 16>(ctx, a) : sort_segments_t<K, kRankOr, 8>(ctx, a);
    if (ctx->rank_mode)
        return big ? sort_segments_t<K, kRankBallot, 16>(ctx, a) : sort_segments_t<K, kRankBallot, 8>(ctx, a);
    return big ? sort_segments_t<K, kRankMatch, 16>(ctx, a) : sort_segments_t<K, kRankMatch, 8>(ctx, a);
}

int sort_segments(fmcs_ctx *ctx, const SortArgs &a)
{
    if (a.n == 0) return FMCS_OK;
    if (a.key_bits == 0 || a.key_bits > 8 * a.bank_bytes)
        return set_error(ctx, FMCS_E_INVAL, "sort: key_bits must be in 1..8*bank_bytes");
    switch (a.bank_bytes) {
    case 2: return sort_dispatch<uint16_t>(ctx, a);
    case 4: return sort_dispatch<uint32_t>(ctx, a);
    case 8: return sort_dispatch<uint64_t>(ctx, a);
    default: return set_error(ctx, FMCS_E_INVAL, "sort: bank_bytes must be 2, 4 or 8");
    }
}

}  // namespace fmcs
