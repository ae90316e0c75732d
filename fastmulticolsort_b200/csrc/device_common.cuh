// device_common.cuh -- device helpers shared by the sm_100a kernels of the
// multi-column sort path: typed key access, radix digits, warp-level
// multi-split ranking (match.any + ballot), and the bounded waits used by the
// decoupled look-back scans (every wait has an iteration limit, after which the
// kernel records FMCS_E_TIMEOUT in a device status word and carries on, so a
// lost predecessor can never hang the GPU).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fmcs {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kWarp = 32;

// Device status word values (mirrors the C-ABI status codes).
constexpr int kDevOk = 0;
constexpr int kDevTimeout = -3;
constexpr int kDevBadInput = -1;

// Look-back words: hi 32 bits = (epoch << 2) | flag, lo 32 bits = value.
constexpr uint32_t kFlagAggregate = 1;
constexpr uint32_t kFlagInclusive = 2;
// A wait gives up after this many polls (with nanosleep back-off that is well
// over a second; a healthy predecessor publishes within microseconds).
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// First statement of every kernel of the library (programmatic dependent
// launch): let the stream's next kernel begin launching now, then wait until
// the previous kernel has completed and its memory is visible.  Both are
// no-ops for a kernel launched without the programmatic attribute.  The next
// kernel is launched only once every block of this one is running, so its
// waiting blocks never keep this one's blocks from being scheduled.
__device__ __forceinline__ void kernel_prologue()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K key, uint32_t lo, uint32_t width)
{
    return (uint32_t)((uint64_t)key >> lo) & ((1u << width) - 1u);
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_volatile_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long lb_word(uint32_t epoch, uint32_t flag, uint32_t value)
{
    return ((unsigned long long)((epoch << 2) | flag) << 32) | value;
}

// Warp-level multi-split rank: for the 32 items of one step (one per lane, in
// lane order), returns each valid item's rank among the warp's items with the
// same digit seen so far, and advances the warp's per-digit counters `whist`.
// Invalid lanes (valid == false) take no rank and leave the counters alone.
// Two ways to find the lanes holding the same digit ("peers"):
//   kRankMatch:  one match.any.sync on the digit;
//   kRankBallot: one ballot per digit bit, peers = AND over bits of the
//                ballot or its complement (the ballot-based multisplit).
//   kRankOr:     (scatter kernels with a per-warp peer array in shared
//                memory) each lane ORs its bit into the word of its digit;
//                after a warp barrier that word is the peer set.  Elsewhere
//                kRankOr ranks as kRankBallot.
constexpr int kRankMatch = 0;
constexpr int kRankBallot = 1;
constexpr int kRankOr = 2;

template <int MODE>
__device__ __forceinline__ uint32_t peers_of(uint32_t digit, bool valid, uint32_t width)
{
    if constexpr (MODE == kRankMatch) {
        return __match_any_sync(0xFFFFFFFFu, valid ? digit : 0xFFFFFFFFu);
    } else {
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
        if (!valid) peers = ~peers;
#pragma unroll
        for (uint32_t b = 0; b < (uint32_t)kRadixBits; ++b) {
            if (b < width) {
                const bool bit = (digit >> b) & 1u;
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
                peers &= bit ? bal : ~bal;
            }
        }
        return peers;
    }
}

template <int MODE = kRankMatch>
__device__ __forceinline__ uint32_t wlms_rank(uint32_t digit, bool valid, uint32_t *whist,
                                              uint32_t width = kRadixBits)
{
    const uint32_t peers = peers_of<MODE>(digit, valid, width);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (valid && lane_id() == leader) {
        base = whist[digit];
        whist[digit] = base + __popc(peers);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    __syncwarp();
    return base + __popc(peers & lanemask_lt());
}

// wlms_rank for a full warp of valid items with full-width (8-bit) digits.
template <int MODE = kRankMatch>
__device__ __forceinline__ uint32_t wlms_rank_full(uint32_t digit, uint32_t *whist)
{
    uint32_t peers;
    if constexpr (MODE == kRankMatch) {
        peers = __match_any_sync(0xFFFFFFFFu, digit);
    } else {
        peers = 0xFFFFFFFFu;
#pragma unroll
        for (uint32_t b = 0; b < (uint32_t)kRadixBits; ++b) {
            const uint32_t bit = (digit >> b) & 1u;
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
            peers &= bit ? bal : ~bal;
        }
    }
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) {
        base = whist[digit];
        whist[digit] = base + __popc(peers);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    __syncwarp();
    return base + __popc(peers & lanemask_lt());
}

// wlms_rank by shared-memory OR: `peerw` is the warp's kRadix-word peer array,
// all zero on entry and left all zero (each digit's leader clears its word).
__device__ __forceinline__ uint32_t wlms_rank_or(uint32_t digit, bool valid, uint32_t *whist, uint32_t *peerw)
{
    const uint32_t lane = lane_id();
    if (valid) atomicOr(&peerw[digit], 1u << lane);
    __syncwarp();
    uint32_t peers = 0, base = 0;
    if (valid) {
        peers = peerw[digit];
        base = whist[digit];
    }
    __syncwarp();
    const uint32_t below = __popc(peers & lanemask_lt());
    if (valid && below == 0) {
        whist[digit] = base + __popc(peers);
        peerw[digit] = 0;
    }
    __syncwarp();
    return base + below;
}

// Exclusive scan of kRadix counters in shared memory by a block of NT threads.
// Returns the total through *total (every thread).  `tmp` holds NT/32 words.
template <int NT>
__device__ __forceinline__ void block_exclusive_scan_radix(uint32_t *cnt, uint32_t *tmp, uint32_t *total)
{
    static_assert(kRadix % NT == 0 || NT % kRadix == 0, "radix/threads");
    constexpr int PER = (kRadix >= NT) ? kRadix / NT : 1;
    const int t = threadIdx.x;
    uint32_t local[PER];
    uint32_t sum = 0;
    if (t * PER < kRadix) {
#pragma unroll
        for (int i = 0; i < PER; ++i) { local[i] = cnt[t * PER + i]; sum += local[i]; }
    }
    // warp inclusive scan of per-thread sums
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane_id() >= o) incl += y;
    }
    const int w = t >> 5;
    if (lane_id() == 31) tmp[w] = incl;
    __syncthreads();
    if (t < 32) {
        uint32_t v = (t < NT / 32) ? tmp[t] : 0;
        uint32_t vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, vi, o);
            if (t >= o) vi += y;
        }
        if (t < NT / 32) tmp[t] = vi - v;  // exclusive warp offsets
        if (t == NT / 32 - 1) tmp[NT / 32] = vi;
    }
    __syncthreads();
    uint32_t run = tmp[w] + incl - sum;
    if (t * PER < kRadix) {
#pragma unroll
        for (int i = 0; i < PER; ++i) { cnt[t * PER + i] = run; run += local[i]; }
    }
    *total = tmp[NT / 32];
    __syncthreads();
}

// Bounded wait on a look-back word of the given epoch.  Returns the word, or 0
// after recording a timeout in *status (the caller treats 0 as an inclusive
// value of 0 so that every waiter still finishes).  `limit` polls at most.
__device__ __forceinline__ unsigned long long lb_wait(const unsigned long long *p, uint32_t epoch,
                                                      int *status, uint32_t limit = kSpinLimit)
{
    uint32_t ns = 16;
    for (uint32_t it = 0; it < limit; ++it) {
        unsigned long long w = ld_volatile_u64(p);
        uint32_t hi = (uint32_t)(w >> 32);
        if ((hi >> 2) == epoch && (hi & 3u) != 0) return w;
        if ((it & 255u) == 255u && *(volatile int *)status != kDevOk) break;
        __nanosleep(ns);
        if (ns < 128) ns <<= 1;
    }
    atomicCAS(status, kDevOk, kDevTimeout);
    return lb_word(epoch, kFlagInclusive, 0);
}

}  // namespace fmcs
