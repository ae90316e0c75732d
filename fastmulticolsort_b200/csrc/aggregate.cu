// aggregate.cu -- per-group aggregates of a payload column: the consumer of
// (order, group) that a GROUP BY query runs next.
//
// The reference stops at (order, group) (Composer::getGroupInfo,
// src/composer.h:59-68); its drivers do not aggregate.  Here, for every sorted
// position i, the payload value of row order[i] joins group group[i]: count,
// sum, min and max per group.  Each thread folds 16 consecutive positions
// (their group ids read as 16-byte vectors), keeping a running aggregate while
// the group id repeats and flushing it with atomics where it changes: after a
// sort plan, whose groups are runs of positions, that is one update per run a
// thread sees; the hash path's last round, whose groups are not runs, costs one
// update per row and is still exact.  Signed payloads are min/max'ed through
// the order-preserving map x ^ 2^63 and mapped back at the end; sums wrap in
// 64 bits (two's complement: the signed sum when no overflow).
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <algorithm>

namespace fmcs {
namespace {

constexpr int kAggItems = 16;
constexpr unsigned long long kSignFlip = 1ull << 63;

__global__ void agg_init_kernel(uint64_t g, unsigned long long *count, unsigned long long *sum,
                                unsigned long long *mn, unsigned long long *mx)
{
    kernel_prologue();
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < g; k += (uint64_t)gridDim.x * blockDim.x) {
        if (count) count[k] = 0;
        if (sum) sum[k] = 0;
        if (mn) mn[k] = ~0ull;
        if (mx) mx[k] = 0;
    }
}

template <typename P>
__device__ __forceinline__ unsigned long long widen(P v, bool is_signed)
{
    // value as 64 bits (sign-extended when signed)
    if constexpr (sizeof(P) == 4) {
        return is_signed ? (unsigned long long)(long long)(int32_t)v : (unsigned long long)(uint32_t)v;
    } else {
        return (unsigned long long)v;
    }
}

__device__ __forceinline__ void flush(uint32_t g, unsigned long long c, unsigned long long s, unsigned long long lo,
                                      unsigned long long hi, unsigned long long *count, unsigned long long *sum,
                                      unsigned long long *mn, unsigned long long *mx)
{
    if (count) atomicAdd(&count[g], c);
    if (sum) atomicAdd(&sum[g], s);
    if (mn) atomicMin(&mn[g], lo);
    if (mx) atomicMax(&mx[g], hi);
}

// Group ids >= ngroups and order entries >= n are not used (they would
// address outside the arrays): they set the status word to bad input.
template <typename P>
__global__ void __launch_bounds__(256) agg_kernel(const P *__restrict__ payload, bool is_signed,
                                                  const uint32_t *__restrict__ order,
                                                  const uint32_t *__restrict__ group, uint64_t n, uint32_t ngroups,
                                                  bool vec, unsigned long long *count, unsigned long long *sum,
                                                  unsigned long long *mn, unsigned long long *mx, int *status)
{
    kernel_prologue();
    const unsigned long long flip = is_signed ? kSignFlip : 0ull;
    const uint64_t chunks = (n + kAggItems - 1) / kAggItems;
    for (uint64_t ch = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; ch < chunks;
         ch += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ch * kAggItems;
        uint32_t gid[kAggItems], row[kAggItems];
        if (vec && i0 + kAggItems <= n) {
            const uint4 *gq = reinterpret_cast<const uint4 *>(group + i0);
            const uint4 *oq = reinterpret_cast<const uint4 *>(order + i0);
#pragma unroll
            for (int w = 0; w < kAggItems / 4; ++w) {
                const uint4 a = gq[w], b = oq[w];
                gid[4 * w] = a.x; gid[4 * w + 1] = a.y; gid[4 * w + 2] = a.z; gid[4 * w + 3] = a.w;
                row[4 * w] = b.x; row[4 * w + 1] = b.y; row[4 * w + 2] = b.z; row[4 * w + 3] = b.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kAggItems; ++k) {
                gid[k] = i0 + k < n ? group[i0 + k] : 0u;
                row[k] = i0 + k < n ? order[i0 + k] : 0u;
            }
        }
        unsigned long long val[kAggItems];
        bool bad = false;
#pragma unroll
        for (int k = 0; k < kAggItems; ++k) {
            const bool in = i0 + k < n && row[k] < n && gid[k] < ngroups;
            bad |= i0 + k < n && !in;
            val[k] = in ? widen<P>(payload[row[k]], is_signed) : 0ull;
        }
        if (bad) {
            atomicCAS(status, kDevOk, kDevBadInput);
            continue;
        }
        uint32_t cur = gid[0];
        unsigned long long c = 0, s = 0, lo = ~0ull, hi = 0;
#pragma unroll
        for (int k = 0; k < kAggItems; ++k) {
            if (i0 + k >= n) break;
            if (gid[k] != cur) {
                flush(cur, c, s, lo, hi, count, sum, mn, mx);
                cur = gid[k];
                c = 0;
                s = 0;
                lo = ~0ull;
                hi = 0;
            }
            const unsigned long long o = val[k] ^ flip;
            c += 1;
            s += val[k];
            lo = o < lo ? o : lo;
            hi = o > hi ? o : hi;
        }
        flush(cur, c, s, lo, hi, count, sum, mn, mx);
    }
}

__global__ void agg_unflip_kernel(uint64_t g, unsigned long long *mn, unsigned long long *mx)
{
    kernel_prologue();
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < g; k += (uint64_t)gridDim.x * blockDim.x) {
        if (mn) mn[k] ^= kSignFlip;
        if (mx) mx[k] ^= kSignFlip;
    }
}

}  // namespace
}  // namespace fmcs

using namespace fmcs;

extern "C" int fmcs_group_aggregate(fmcs_ctx *ctx, const void *payload, uint32_t payload_bytes, int is_signed,
                                    const uint32_t *order, const uint32_t *group, uint64_t n, uint32_t ngroups,
                                    uint64_t *count, uint64_t *sum, uint64_t *min, uint64_t *max)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!(payload_bytes == 4 || payload_bytes == 8))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_group_aggregate: payload_bytes must be 4 or 8");
    if (n && (!payload || !order || !group))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_group_aggregate: payload, order and group are required");
    if (n && ngroups == 0) return set_error(ctx, FMCS_E_INVAL, "fmcs_group_aggregate: ngroups must be > 0");
    for (const void *p : {payload, (const void *)order, (const void *)group, (const void *)count, (const void *)sum,
                          (const void *)min, (const void *)max})
        if (p && !is_device_ptr(p))
            return set_error(ctx, FMCS_E_INVAL, "fmcs_group_aggregate: arrays must be device memory");
    unsigned long long *c = (unsigned long long *)count, *s = (unsigned long long *)sum;
    unsigned long long *lo = (unsigned long long *)min, *hi = (unsigned long long *)max;
    cudaStream_t st = ctx->stream;
    const unsigned ig = (unsigned)std::min<uint64_t>((ngroups + 255) / 256, (uint64_t)ctx->num_sms * 8);
    if (ngroups) {
        LaunchScope ls_(ctx, "agg_init");
        launch_k(agg_init_kernel, ig ? ig : 1, 256, 0, st, ngroups, c, s, lo, hi);
    }
    if (n) {
        const uint64_t chunks = (n + kAggItems - 1) / kAggItems;
        const unsigned grid = (unsigned)std::min<uint64_t>((chunks + 255) / 256, (uint64_t)ctx->num_sms * 16);
        const bool vec = (((uintptr_t)order | (uintptr_t)group) & 15u) == 0;
        LaunchScope ls_(ctx, "aggregate");
        if (payload_bytes == 4)
            launch_k(agg_kernel<uint32_t>, grid, 256, 0, st, (const uint32_t *)payload, is_signed != 0, order, group, n,
                                                       ngroups, vec, c, s, lo, hi, ctx->d_status);
        else
            launch_k(agg_kernel<uint64_t>, grid, 256, 0, st, (const uint64_t *)payload, is_signed != 0, order, group, n,
                                                       ngroups, vec, c, s, lo, hi, ctx->d_status);
    }
    if (is_signed && ngroups && (lo || hi)) {
        LaunchScope ls_(ctx, "agg_unflip");
        launch_k(agg_unflip_kernel, ig ? ig : 1, 256, 0, st, ngroups, lo, hi);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_group_aggregate launch");
    return check_status(ctx, "fmcs_group_aggregate");
}
