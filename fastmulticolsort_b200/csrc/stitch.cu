// stitch.cu -- (a) bit stitching of one bank in ONE pass.
//
// The reference builds a bank slice by slice with whole-column AVX2 passes:
// ShiftLeftBatch shifts the bank left by the next slice's width, then
// AssembleFromColumn ORs in (src >> (origW - end)) & mask
// (src/column.h:105-180, 208-1060; loop at src/stitch_composer.cpp:655-703).
// That reads and writes the bank once per slice.  Here every thread owns four
// consecutive rows, reads each source slice with one vector load per row
// group, folds the slices in registers and writes the bank once: the kernel
// moves exactly sum(source bytes) + bank bytes per row.
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <algorithm>

namespace fmcs {

namespace {

struct StitchParams {
    StitchSlice s[kMaxSlices];
    int ns;
};

__device__ __forceinline__ void load4(const void *base, uint32_t bytes, uint64_t row, bool vec,
                                      uint64_t n, uint64_t v[4])
{
    if (vec) {
        switch (bytes) {
        case 1: {
            uint32_t x = *reinterpret_cast<const uint32_t *>((const uint8_t *)base + row);
            v[0] = x & 0xFF; v[1] = (x >> 8) & 0xFF; v[2] = (x >> 16) & 0xFF; v[3] = x >> 24;
            return;
        }
        case 2: {
            uint2 x = *reinterpret_cast<const uint2 *>((const uint16_t *)base + row);
            v[0] = x.x & 0xFFFF; v[1] = x.x >> 16; v[2] = x.y & 0xFFFF; v[3] = x.y >> 16;
            return;
        }
        case 4: {
            uint4 x = *reinterpret_cast<const uint4 *>((const uint32_t *)base + row);
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
            return;
        }
        default: {
            const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>((const uint64_t *)base + row);
            ulonglong2 a = p[0], b = p[1];
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
            return;
        }
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint64_t r = row + k;
        if (r >= n) { v[k] = 0; continue; }
        switch (bytes) {
        case 1: v[k] = ((const uint8_t *)base)[r]; break;
        case 2: v[k] = ((const uint16_t *)base)[r]; break;
        case 4: v[k] = ((const uint32_t *)base)[r]; break;
        default: v[k] = ((const uint64_t *)base)[r]; break;
        }
    }
}

template <typename B>
__device__ __forceinline__ void store4(B *bank, uint64_t row, bool vec, uint64_t n, const uint64_t a[4])
{
    if (vec) {
        if constexpr (sizeof(B) == 1) {
            uint32_t x = (uint32_t)(a[0] & 0xFF) | (uint32_t)(a[1] & 0xFF) << 8 |
                         (uint32_t)(a[2] & 0xFF) << 16 | (uint32_t)(a[3] & 0xFF) << 24;
            *reinterpret_cast<uint32_t *>(bank + row) = x;
        } else if constexpr (sizeof(B) == 2) {
            uint2 x;
            x.x = (uint32_t)(a[0] & 0xFFFF) | (uint32_t)(a[1] & 0xFFFF) << 16;
            x.y = (uint32_t)(a[2] & 0xFFFF) | (uint32_t)(a[3] & 0xFFFF) << 16;
            *reinterpret_cast<uint2 *>(bank + row) = x;
        } else if constexpr (sizeof(B) == 4) {
            *reinterpret_cast<uint4 *>(bank + row) =
                make_uint4((uint32_t)a[0], (uint32_t)a[1], (uint32_t)a[2], (uint32_t)a[3]);
        } else {
            ulonglong2 *p = reinterpret_cast<ulonglong2 *>(bank + row);
            p[0] = make_ulonglong2(a[0], a[1]);
            p[1] = make_ulonglong2(a[2], a[3]);
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (row + k < n) bank[row + k] = (B)a[k];
}

// With top_hist the kernel also counts the first radix level's digits, one
// 256-word row per chunk of 2^chunk_shift rows and, after them, one row for
// the whole bank; each CTA then takes a contiguous
// range of block_groups groups of 4 rows (at most one chunk long, so that it
// meets at most two chunks, counted in two shared histograms).  Without, the
// groups are spread grid-stride.
template <typename B>
__global__ void __launch_bounds__(256, 4) stitch_kernel(const __grid_constant__ StitchParams p, B *bank,
                                                     uint64_t n, bool aligned, uint32_t *top_hist,
                                                     uint32_t hist_lo, uint32_t hist_mask, uint32_t chunk_shift,
                                                     uint64_t block_groups)
{
    kernel_prologue();
    __shared__ uint32_t sh[2][256];
    const uint64_t groups = (n + 3) / 4;
    // this CTA's groups: [g_begin, g_end), `stride` apart per thread step
    uint64_t g_begin = blockIdx.x * (uint64_t)blockDim.x, g_end = groups;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t chunk0 = 0;   // the chunk of the CTA's first row
    if (top_hist) {
        for (int d = threadIdx.x; d < 2 * 256; d += blockDim.x) (&sh[0][0])[d] = 0;
        __syncthreads();
        g_begin = blockIdx.x * block_groups;
        g_end = min(groups, g_begin + block_groups);
        stride = blockDim.x;
        chunk0 = (g_begin * 4) >> chunk_shift;
    }
    // Each thread takes two groups of 4 rows per step (a stride apart), so
    // that the loads of both are in flight together.
    for (uint64_t g = g_begin + threadIdx.x; g < g_end; g += 2 * stride) {
        const bool two = g + stride < g_end;
        const uint64_t row0 = g * 4, row1 = (g + stride) * 4;
        const bool vec0 = aligned && row0 + 4 <= n;
        const bool vec1 = aligned && row1 + 4 <= n;
        uint64_t acc0[4] = {0, 0, 0, 0}, acc1[4] = {0, 0, 0, 0};
        for (int s = 0; s < p.ns; ++s) {
            const StitchSlice sl = p.s[s];
            uint64_t v0[4], v1[4] = {0, 0, 0, 0};
            load4(sl.src, sl.src_bytes, row0, vec0, n, v0);
            if (two) load4(sl.src, sl.src_bytes, row1, vec1, n, v1);
            const uint64_t mask = sl.width >= 64 ? ~0ull : ((1ull << sl.width) - 1);
            const uint64_t flip = sl.invert ? mask : 0ull;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint64_t x0 = ((v0[k] >> sl.rshift) & mask) ^ flip;
                const uint64_t x1 = ((v1[k] >> sl.rshift) & mask) ^ flip;
                acc0[k] = (s == 0 || sl.width >= 64) ? x0 : ((acc0[k] << sl.width) | x0);
                acc1[k] = (s == 0 || sl.width >= 64) ? x1 : ((acc1[k] << sl.width) | x1);
            }
        }
        store4<B>(bank, row0, vec0, n, acc0);
        if (two) store4<B>(bank, row1, vec1, n, acc1);
        if (top_hist) {
            // a group's 4 rows share a chunk (chunks are at least 4 rows)
            uint32_t *h0 = sh[(row0 >> chunk_shift) - chunk0];
            uint32_t *h1 = two ? sh[(row1 >> chunk_shift) - chunk0] : h0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (row0 + k < n) atomicAdd(&h0[(uint32_t)(acc0[k] >> hist_lo) & hist_mask], 1u);
                if (two && row1 + k < n) atomicAdd(&h1[(uint32_t)(acc1[k] >> hist_lo) & hist_mask], 1u);
            }
        }
    }
    if (top_hist) {
        __syncthreads();
        const uint64_t nchunks = ((n - 1) >> chunk_shift) + 1;
        for (int i = threadIdx.x; i < 2 * 256; i += blockDim.x) {
            const uint64_t c = chunk0 + (uint64_t)(i >> 8);
            const uint32_t v = (&sh[0][0])[i];
            if (v && c < nchunks) atomicAdd(&top_hist[c * 256 + (i & 255)], v);
        }
        // and the whole bank's histogram, the row after the chunks' rows
        for (int d = threadIdx.x; d < 256; d += blockDim.x) {
            const uint32_t v = sh[0][d] + sh[1][d];
            if (v) atomicAdd(&top_hist[nchunks * 256 + d], v);
        }
    }
}

// Slice-at-a-time primitives (the reference's ShiftLeftBatch / AssembleFromColumn).
template <typename B>
__global__ void __launch_bounds__(256) bank_update_kernel(B *bank, uint64_t n, uint32_t lshift, const void *src,
                                                          uint32_t src_bytes, uint32_t rshift, uint32_t width)
{
    kernel_prologue();
    const uint64_t mask = width >= 64 ? ~0ull : ((1ull << width) - 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!src) {
            bank[i] = lshift >= 8 * sizeof(B) ? B(0) : (B)((uint64_t)bank[i] << lshift);
        } else {
            uint64_t v;
            switch (src_bytes) {
            case 1: v = ((const uint8_t *)src)[i]; break;
            case 2: v = ((const uint16_t *)src)[i]; break;
            case 4: v = ((const uint32_t *)src)[i]; break;
            default: v = ((const uint64_t *)src)[i]; break;
            }
            bank[i] = (B)((uint64_t)bank[i] | ((v >> rshift) & mask));
        }
    }
}

}  // namespace

int launch_bank_update(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n, uint32_t lshift,
                       const void *src, uint32_t src_bytes, uint32_t rshift, uint32_t width)
{
    if (n == 0) return FMCS_OK;
    const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 8);
    LaunchScope ls_(ctx, src ? "assemble" : "shift_left");
    switch (bank_bytes) {
    case 1: launch_k(bank_update_kernel<uint8_t>, grid, 256, 0, ctx->stream,
                     (uint8_t *)bank, n, lshift, src, src_bytes, rshift, width); break;
    case 2: launch_k(bank_update_kernel<uint16_t>, grid, 256, 0, ctx->stream,
                     (uint16_t *)bank, n, lshift, src, src_bytes, rshift, width); break;
    case 4: launch_k(bank_update_kernel<uint32_t>, grid, 256, 0, ctx->stream,
                     (uint32_t *)bank, n, lshift, src, src_bytes, rshift, width); break;
    case 8: launch_k(bank_update_kernel<uint64_t>, grid, 256, 0, ctx->stream,
                     (uint64_t *)bank, n, lshift, src, src_bytes, rshift, width); break;
    default: return set_error(ctx, FMCS_E_INVAL, "bank_bytes must be 1, 2, 4 or 8");
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "bank update launch");
}

int launch_stitch(fmcs_ctx *ctx, const StitchSlice *sl, int ns, void *bank, uint32_t bank_bytes,
                  uint64_t n, uint32_t *top_hist, uint32_t key_bits, uint32_t chunk_rows, cudaStream_t stream)
{
    cudaStream_t st = stream ? stream : ctx->stream;
    if (ns < 1 || ns > kMaxSlices) return set_error(ctx, FMCS_E_INVAL, "stitch: 1..32 slices");
    if (!(bank_bytes == 1 || bank_bytes == 2 || bank_bytes == 4 || bank_bytes == 8))
        return set_error(ctx, FMCS_E_INVAL, "stitch: bank_bytes must be 1, 2, 4 or 8");
    if (n == 0) return FMCS_OK;
    StitchParams p;
    bool aligned = ((uintptr_t)bank % 16) == 0;
    for (int i = 0; i < ns; ++i) {
        p.s[i] = sl[i];
        aligned = aligned && ((uintptr_t)sl[i].src % 16) == 0;
    }
    p.ns = ns;
    const uint64_t groups = (n + 3) / 4;
    uint64_t blocks = (groups + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->num_sms * 8;
    if (blocks > cap) blocks = cap;
    uint32_t hist_lo = 0, hist_mask = 0;
    uint64_t block_groups = 0;
    uint32_t chunk_shift = 0;
    if (top_hist) {
        if (chunk_rows < 4 || (chunk_rows & (chunk_rows - 1)))
            return set_error(ctx, FMCS_E_INVAL, "stitch: chunk rows must be a power of two >= 4");
        chunk_shift = (uint32_t)__builtin_ctz(chunk_rows);
        const uint32_t width = key_bits < 8u ? key_bits : 8u;
        hist_lo = key_bits - width;
        hist_mask = (1u << width) - 1u;
        const uint64_t nchunks = (n + chunk_rows - 1) / chunk_rows;
        cudaMemsetAsync(top_hist, 0, (nchunks + 1) * 256 * sizeof(uint32_t), st);
        // contiguous ranges of whole 256-group steps, at most one chunk each
        block_groups = (groups + blocks - 1) / blocks;
        block_groups = (block_groups + 255) / 256 * 256;
        const uint64_t chunk_groups = chunk_rows / 4;
        if (block_groups > chunk_groups) block_groups = chunk_groups;
        blocks = (groups + block_groups - 1) / block_groups;
    }
    const unsigned grid = (unsigned)blocks;
    LaunchScope ls_(ctx, "stitch");
    switch (bank_bytes) {
    case 1:
        launch_k(stitch_kernel<uint8_t>, grid, 256, 0, st,
                 p, (uint8_t *)bank, n, aligned, top_hist, hist_lo, hist_mask, chunk_shift, block_groups);
        break;
    case 2:
        launch_k(stitch_kernel<uint16_t>, grid, 256, 0, st,
                 p, (uint16_t *)bank, n, aligned, top_hist, hist_lo, hist_mask, chunk_shift, block_groups);
        break;
    case 4:
        launch_k(stitch_kernel<uint32_t>, grid, 256, 0, st,
                 p, (uint32_t *)bank, n, aligned, top_hist, hist_lo, hist_mask, chunk_shift, block_groups);
        break;
    case 8:
        launch_k(stitch_kernel<uint64_t>, grid, 256, 0, st,
                 p, (uint64_t *)bank, n, aligned, top_hist, hist_lo, hist_mask, chunk_shift, block_groups);
        break;
    default: return set_error(ctx, FMCS_E_INVAL, "stitch: bank_bytes must be 1, 2, 4 or 8");
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "stitch launch");
}

}  // namespace fmcs
