// gather.cu -- (c) out[i] = bank[order[i]] (Composer::BATproject,
// src/composer.cpp:608-628).  The sort rounds fuse this gather into their
// first read (segsort.cu, the EXT source); this standalone kernel backs the
// fmcs_gather entry point.  Each thread issues 8 independent gathers before it
// stores, so enough random reads are in flight to cover HBM latency.
#include "device_common.cuh"
#include "fmcs_internal.h"

namespace fmcs {

namespace {

constexpr int kGatherItems = 8;

template <typename T>
__global__ void __launch_bounds__(256) gather_kernel(const T *__restrict__ bank, const uint32_t *__restrict__ order,
                                                     T *__restrict__ out, uint64_t n)
{
    kernel_prologue();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base < n;
         base += stride * kGatherItems) {
        uint32_t idx[kGatherItems];
        T v[kGatherItems];
#pragma unroll
        for (int j = 0; j < kGatherItems; ++j) {
            const uint64_t i = base + j * stride;
            idx[j] = i < n ? order[i] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kGatherItems; ++j) {
            const uint64_t i = base + j * stride;
            v[j] = i < n ? bank[idx[j]] : T(0);
        }
#pragma unroll
        for (int j = 0; j < kGatherItems; ++j) {
            const uint64_t i = base + j * stride;
            if (i < n) out[i] = v[j];
        }
    }
}

}  // namespace

int launch_gather(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, const uint32_t *order, void *out,
                  uint64_t n)
{
    if (n == 0) return FMCS_OK;
    const unsigned grid = (unsigned)ctx->num_sms * 8;
    switch (bank_bytes) {
    case 1: { LaunchScope ls_(ctx, "gather");
        launch_k(gather_kernel<uint8_t>, grid, 256, 0, ctx->stream, (const uint8_t *)bank, order, (uint8_t *)out, n);
    } break;
    case 2: { LaunchScope ls_(ctx, "gather");
        launch_k(gather_kernel<uint16_t>, grid, 256, 0, ctx->stream, (const uint16_t *)bank, order, (uint16_t *)out, n);
    } break;
    case 4: { LaunchScope ls_(ctx, "gather");
        launch_k(gather_kernel<uint32_t>, grid, 256, 0, ctx->stream, (const uint32_t *)bank, order, (uint32_t *)out, n);
    } break;
    case 8: { LaunchScope ls_(ctx, "gather");
        launch_k(gather_kernel<uint64_t>, grid, 256, 0, ctx->stream, (const uint64_t *)bank, order, (uint64_t *)out, n);
    } break;
    default: return set_error(ctx, FMCS_E_INVAL, "gather: bank_bytes must be 1, 2, 4 or 8");
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "gather launch");
}

}  // namespace fmcs
