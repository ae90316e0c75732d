// scan.cu -- (d) group-boundary scan and segment extraction, one pass each.
//
// Reference: Composer::extractGroupInfo<T> (src/composer.cpp:630-678) computes
//   g[0] = 0;  g[i] = g[i-1] + (v[i] != v[i-1] || in[i] != in[i-1])
// with a scalar loop.  Here one kernel reads each key (and in_group word) once:
// adjacent difference -> warp ballot -> popc prefix -> block scan -> decoupled
// look-back across tiles (bounded waits) -> dense ids.  The same kernel, given
// only in_group, emits the start position of every run of equal in_group (the
// segments that the next round sorts; the reference finds them with a scalar
// walk, src/composer.cpp:1280-1335).
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <mutex>

namespace fmcs {

namespace {

constexpr int kScanThreads = 512;              // a tile of 8192 positions: half as many look-back steps
constexpr int kScanItems = 16;                  // per thread
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kScanWarps = kScanThreads / 32;

// kScanItems consecutive values starting at i0 (zero past n); 16-byte vector
// loads when the run is whole and VEC (the caller checked the alignment).
template <typename T, bool VEC>
__device__ __forceinline__ void load_run(const T *__restrict__ p, uint64_t i0, uint64_t n, T (&v)[kScanItems])
{
    if (VEC && i0 + kScanItems <= n) {
        constexpr int W = kScanItems * (int)sizeof(T) / 16;
        const uint4 *q = reinterpret_cast<const uint4 *>(p + i0);
        uint4 t[W];
#pragma unroll
        for (int w = 0; w < W; ++w) t[w] = q[w];
        memcpy(&v[0], &t[0], sizeof(t));
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = i0 + k < n ? p[i0 + k] : T(0);
    }
}

// Decoupled look-back by one warp: each lane reads one predecessor's word
// (bounded waits), and the warp adds the aggregates back to the nearest
// inclusive prefix.  Returns the exclusive prefix of `tile` (every lane).
__device__ __forceinline__ uint32_t warp_lookback(unsigned long long *lookback, uint32_t tile, uint32_t epoch,
                                                  int *status)
{
    const int lane = threadIdx.x & 31;
    uint32_t excl = 0;
    int64_t last = (int64_t)tile - 1;   // the window is tiles last - lane
    for (;;) {
        const int64_t p = last - lane;
        const unsigned long long w = p >= 0 ? lb_wait(&lookback[p], epoch, status) : lb_word(epoch, kFlagInclusive, 0);
        const uint32_t inc = __ballot_sync(0xFFFFFFFFu, ((uint32_t)(w >> 32) & 3u) == kFlagInclusive);
        const int first = inc ? __ffs(inc) - 1 : 32;   // nearest inclusive predecessor
        uint32_t v = lane <= first ? (uint32_t)w : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        excl += v;
        if (inc) return excl;
        last -= 32;
    }
}

// One tile of kScanTile positions per block; thread t owns the kScanItems
// consecutive positions starting at tile base + t * kScanItems.
template <typename K, bool VEC>
__global__ void __launch_bounds__(kScanThreads)
boundary_scan_kernel(const K *__restrict__ keys, const uint32_t *__restrict__ in_group,
                     const uint8_t *__restrict__ flags, uint32_t *__restrict__ out_group, uint32_t *__restrict__ seg_start,
                     uint64_t n, uint32_t *tile_counter, unsigned long long *lookback,
                     uint32_t epoch, uint32_t *d_count, int *status)
{
    kernel_prologue();
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kScanWarps + 1];
    __shared__ uint32_t s_excl;

    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kScanTile;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t i0 = base + (uint64_t)threadIdx.x * kScanItems;

    // boundary flags of the thread's positions, bit k = position i0 + k
    uint32_t fl = 0;
    if (i0 < n) {
        if (flags) {
            uint8_t f[kScanItems];
            load_run<uint8_t, VEC>(flags, i0, n, f);
#pragma unroll
            for (int k = 0; k < kScanItems; ++k) fl |= (uint32_t)(f[k] != 0) << k;
        } else {
            if (keys) {
                K v[kScanItems];
                load_run<K, VEC>(keys, i0, n, v);
                K prev = i0 > 0 ? keys[i0 - 1] : K(0);
#pragma unroll
                for (int k = 0; k < kScanItems; ++k) {
                    fl |= (uint32_t)(v[k] != prev) << k;
                    prev = v[k];
                }
            }
            if (in_group) {
                uint32_t g[kScanItems];
                load_run<uint32_t, VEC>(in_group, i0, n, g);
                uint32_t prev = i0 > 0 ? in_group[i0 - 1] : 0u;
#pragma unroll
                for (int k = 0; k < kScanItems; ++k) {
                    fl |= (uint32_t)(g[k] != prev) << k;
                    prev = g[k];
                }
            }
            if (i0 == 0) fl |= 1u;
        }
        if (n - i0 < (uint64_t)kScanItems) fl &= (1u << (uint32_t)(n - i0)) - 1u;   // positions past n
    }
    const uint32_t cnt = __popc(fl);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t wv = lane < kScanWarps ? s_warp[lane] : 0u;
        uint32_t wi = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += y;
        }
        const uint32_t agg = __shfl_sync(0xFFFFFFFFu, wi, kScanWarps - 1);
        if (lane < kScanWarps) s_warp[lane] = wi - wv;
        uint32_t excl = 0;
        if (tile == 0) {
            if (lane == 0) st_volatile_u64(&lookback[0], lb_word(epoch, kFlagInclusive, agg));
        } else {
            if (lane == 0) st_volatile_u64(&lookback[tile], lb_word(epoch, kFlagAggregate, agg));
            excl = warp_lookback(lookback, tile, epoch, status);
            if (lane == 0) st_volatile_u64(&lookback[tile], lb_word(epoch, kFlagInclusive, excl + agg));
        }
        if (lane == 0) {
            s_excl = excl;
            s_warp[kScanWarps] = agg;
            if (base + kScanTile >= n && d_count) *d_count = excl + agg;  // the last tile
        }
    }
    __syncthreads();
    if (i0 < n) {
        // 1-based id of the group holding position i0 + k, for every k
        uint32_t id = s_excl + s_warp[warp] + incl - cnt;
        if (out_group) {
            uint32_t o[kScanItems];
#pragma unroll
            for (int k = 0; k < kScanItems; ++k) {
                id += (fl >> k) & 1u;
                o[k] = id - 1u;
            }
            if (VEC && i0 + kScanItems <= n) {
                uint4 *q = reinterpret_cast<uint4 *>(out_group + i0);
#pragma unroll
                for (int w = 0; w < kScanItems / 4; ++w) q[w] = make_uint4(o[4 * w], o[4 * w + 1], o[4 * w + 2], o[4 * w + 3]);
            } else {
#pragma unroll
                for (int k = 0; k < kScanItems; ++k)
                    if (i0 + k < n) out_group[i0 + k] = o[k];
            }
        }
        if (seg_start) {
            uint32_t sid = s_excl + s_warp[warp] + incl - cnt;
            for (uint32_t m = fl; m; m &= m - 1) {
                const uint32_t k = __ffs(m) - 1;
                seg_start[sid++] = (uint32_t)(i0 + k);
            }
        }
    }
    if (seg_start && base + kScanTile >= n && threadIdx.x == 0) {
        // the end sentinel after the last segment
        seg_start[s_excl + s_warp[kScanWarps]] = (uint32_t)n;
    }
}

// Launches the scan, with 16-byte vector accesses when every array allows.
template <typename K>
void launch_scan(unsigned grid, cudaStream_t st, const K *keys, const uint32_t *in_group, const uint8_t *flags,
                 uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *tile_counter,
                 unsigned long long *lookback, uint32_t epoch, uint32_t *d_count, int *status)
{
    const bool vec = (((uintptr_t)keys | (uintptr_t)in_group | (uintptr_t)flags | (uintptr_t)out_group) & 15u) == 0;
    if (vec)
        launch_k(boundary_scan_kernel<K, true>, grid, kScanThreads, 0, st,
                 keys, in_group, flags, out_group, seg_start, n,
                                                                      tile_counter, lookback, epoch, d_count, status);
    else
        launch_k(boundary_scan_kernel<K, false>, grid, kScanThreads, 0, st,
                 keys, in_group, flags, out_group, seg_start, n,
                                                                       tile_counter, lookback, epoch, d_count, status);
}

int run_boundary_scan(fmcs_ctx *ctx, const void *keys, uint32_t key_bytes, const uint32_t *in_group,
                      const uint8_t *flags, uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *d_count)
{
    if (n == 0) {
        if (d_count) cudaMemsetAsync(d_count, 0, sizeof(uint32_t), ctx->stream);
        if (seg_start) cudaMemsetAsync(seg_start, 0, sizeof(uint32_t), ctx->stream);
        return FMCS_OK;
    }
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    void *lb = nullptr, *cnt = nullptr;
    int rc = ws_get(ctx, kSlotScanTiles, tiles * sizeof(unsigned long long), &lb, true);
    if (rc) return rc;
    rc = ws_get(ctx, kSlotCounters, 4096, &cnt);
    if (rc) return rc;
    uint32_t *tile_counter = (uint32_t *)cnt;  // word 0 of the counters slot
    cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), ctx->stream);
    const uint32_t epoch = ctx->epoch++;
    const unsigned grid = (unsigned)tiles;
    unsigned long long *lbw = (unsigned long long *)lb;
    LaunchScope ls_(ctx, "boundary_scan");
    switch (keys ? key_bytes : 0) {
    case 0:
        launch_scan<uint32_t>(grid, ctx->stream, nullptr, in_group, flags, out_group, seg_start, n, tile_counter, lbw,
                              epoch, d_count, ctx->d_status);
        break;
    case 1:
        launch_scan<uint8_t>(grid, ctx->stream, (const uint8_t *)keys, in_group, flags, out_group, seg_start, n,
                             tile_counter, lbw, epoch, d_count, ctx->d_status);
        break;
    case 2:
        launch_scan<uint16_t>(grid, ctx->stream, (const uint16_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_counter, lbw, epoch, d_count, ctx->d_status);
        break;
    case 4:
        launch_scan<uint32_t>(grid, ctx->stream, (const uint32_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_counter, lbw, epoch, d_count, ctx->d_status);
        break;
    case 8:
        launch_scan<uint64_t>(grid, ctx->stream, (const uint64_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_counter, lbw, epoch, d_count, ctx->d_status);
        break;
    default:
        return set_error(ctx, FMCS_E_INVAL, "boundary scan: bad key width");
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "boundary scan launch");
}

}  // namespace

int launch_group_ids(fmcs_ctx *ctx, const void *keys, uint32_t key_bytes, const uint32_t *in_group,
                     uint32_t *out_group, uint64_t n, uint32_t *d_ngroups)
{
    return run_boundary_scan(ctx, keys, key_bytes, in_group, nullptr, out_group, nullptr, n, d_ngroups);
}

int launch_segments(fmcs_ctx *ctx, const uint32_t *in_group, uint32_t *seg_start, uint32_t *d_nseg,
                    uint64_t n)
{
    return run_boundary_scan(ctx, nullptr, 0, in_group, nullptr, nullptr, seg_start, n, d_nseg);
}

int launch_group_ids_segments(fmcs_ctx *ctx, const void *keys, uint32_t key_bytes, const uint32_t *in_group,
                              uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *d_count)
{
    return run_boundary_scan(ctx, keys, key_bytes, in_group, nullptr, out_group, seg_start, n, d_count);
}

namespace {
__global__ void iota_kernel(uint32_t *v, uint64_t n)
{
    kernel_prologue();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}
}  // namespace

int launch_iota(fmcs_ctx *ctx, uint32_t *v, uint64_t n)
{
    if (n == 0) return FMCS_OK;
    { LaunchScope ls_(ctx, "iota");
        launch_k(iota_kernel, ctx->num_sms * 8, 256, 0, ctx->stream, v, n);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "iota launch");
}

int launch_flag_rank(fmcs_ctx *ctx, const uint8_t *flags, uint32_t *rank, uint64_t n, uint32_t *d_count)
{
    return run_boundary_scan(ctx, nullptr, 0, nullptr, flags, rank, nullptr, n, d_count);
}

}  // namespace fmcs

// ---------------------------------------------------------------------------
// Allocation-free group ids.
//
// Some callers cannot let a library allocate device memory: query engines
// that reserve all of HBM up front in their own pool (a cudaMalloc from inside
// the library would fail or fragment that pool), and latency-critical callers
// that cannot afford the device-wide synchronization that cudaMalloc/cudaFree
// imply.  fmcs_group_ids_noalloc serves them: the same one-pass boundary scan
// as the group ids of a sort round, with its scratch (the decoupled look-back
// words, the tile counter, the group count and the wait status) in the
// file-scope device array below instead of the context's workspace.  The
// caller passes device inputs and outputs; no context is needed.
//
// The array is modest (kNoAllocTiles look-back words, 128 KiB) and every GPU
// that loads the library holds it until the process exits.  n is bounded at
// 67,108,864 rows (at most 8,192 scan tiles).  All calls share it and it keeps the
// last call's contents, so each call clears the words that must start at zero;
// calls whose work overlaps on the GPU (two streams, or two host threads)
// race on it and must be serialized by the caller.
// ---------------------------------------------------------------------------
namespace fmcs {
namespace {

constexpr uint64_t kNoAllocTiles = 16384;
constexpr uint64_t kNoAllocMaxRows = 67108864;
static_assert(kNoAllocMaxRows / kScanTile <= kNoAllocTiles, "look-back words for every tile");
// layout (64-bit words): [0, kNoAllocTiles) look-back; then the tile counter,
// the group count and the status word, one 64-bit word each
constexpr uint64_t kNoAllocWords = kNoAllocTiles + 4;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long *g_noalloc_ptr[kMaxDevices] = {};

// Host code cannot use g_noalloc_scratch's name as a device address: resolve
// the device address once per device, with that device current.
int noalloc_scratch(unsigned long long **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FMCS_E_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return FMCS_E_CUDA;
        }
        g_noalloc_ptr[dev] = (unsigned long long *)p;
    }
    *out = g_noalloc_ptr[dev];
    return FMCS_OK;
}

}  // namespace

}  // namespace fmcs

extern "C" int fmcs_group_ids_noalloc(void *stream, const void *keys, uint32_t key_bytes,
                                      const uint32_t *in_group, uint32_t *out_group, uint64_t n,
                                      uint32_t *ngroups)
{
    using namespace fmcs;
    if (ngroups) *ngroups = 0;
    if (!(key_bytes == 1 || key_bytes == 2 || key_bytes == 4 || key_bytes == 8)) return FMCS_E_INVAL;
    if (n > kNoAllocMaxRows) return FMCS_E_INVAL;   // beyond the static scratch: 67,108,864 rows
    if (n == 0) return FMCS_OK;
    if (!keys || !out_group || !is_device_ptr(keys) || !is_device_ptr(out_group) ||
        (in_group && !is_device_ptr(in_group)))
        return FMCS_E_INVAL;   // device pointers only: staging host data would allocate
    unsigned long long *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    unsigned long long *lookback = scratch;
    uint32_t *tile_counter = (uint32_t *)(scratch + kNoAllocTiles);
    uint32_t *d_count = (uint32_t *)(scratch + kNoAllocTiles + 1);
    int *status = (int *)(scratch + kNoAllocTiles + 2);
    // the previous call's words: look-back of the tiles this call uses, counter,
    // count and status all start at zero
    cudaError_t e = cudaMemsetAsync(lookback, 0, tiles * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(tile_counter, 0, 3 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return FMCS_E_CUDA;
    const uint32_t epoch = 1;
    const unsigned grid = (unsigned)tiles;
    switch (key_bytes) {
    case 1:
        launch_scan<uint8_t>(grid, st, (const uint8_t *)keys, in_group, nullptr, out_group, nullptr, n,
                             tile_counter, lookback, epoch, d_count, status);
        break;
    case 2:
        launch_scan<uint16_t>(grid, st, (const uint16_t *)keys, in_group, nullptr, out_group, nullptr, n,
                              tile_counter, lookback, epoch, d_count, status);
        break;
    case 4:
        launch_scan<uint32_t>(grid, st, (const uint32_t *)keys, in_group, nullptr, out_group, nullptr, n,
                              tile_counter, lookback, epoch, d_count, status);
        break;
    default:
        launch_scan<uint64_t>(grid, st, (const uint64_t *)keys, in_group, nullptr, out_group, nullptr, n,
                              tile_counter, lookback, epoch, d_count, status);
        break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return FMCS_E_CUDA;
    // read the count and the wait status back (into the caller's stack: no
    // allocation) and finish the call
    uint32_t back[3] = {0, 0, 0};
    e = cudaMemcpyAsync(back, d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(back + 1, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return FMCS_E_CUDA;
    if ((int)back[1] == kDevTimeout) return FMCS_E_TIMEOUT;
    if (back[1] != 0) return FMCS_E_CUDA;
    if (ngroups) *ngroups = back[0];
    return FMCS_OK;
}
