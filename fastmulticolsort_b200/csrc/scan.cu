// scan.cu -- (d) group-boundary scan and segment extraction.
//
// Reference: Composer::extractGroupInfo<T> (src/composer.cpp:630-678) computes
//   g[0] = 0;  g[i] = g[i-1] + (v[i] != v[i-1] || in[i] != in[i-1])
// with a scalar loop.  Here, in three launches with no waits between blocks:
// (1) every tile of 8192 positions counts its group starts (adjacent
// difference -> per-lane bit masks -> popc) and stores the masks (2 bytes per
// 16 rows), (2) one block scans the tile counts, (3) every tile reads its
// masks back and writes dense ids from its prefix (warp and block scans inside
// the tile).  The keys are read once.  (The allocation-free entry point has no
// room for the masks: its pass 3 recomputes them from the keys, last tile
// first, so that the keys (1) read last are still in L2.)  The same kernels, given only in_group,
// emit the start position of every run of equal in_group (the segments that
// the next round sorts; the reference finds them with a scalar walk,
// src/composer.cpp:1280-1335).
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <algorithm>
#include <mutex>

namespace fmcs {

namespace {

constexpr int kScanThreads = 512;              // a tile of 8192 positions
constexpr int kScanItems = 16;                  // per thread
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kScanWarps = kScanThreads / 32;

// P consecutive values of a starting at p (zero past n), as one 4-, 8- or
// 16-byte-multiple vector load when VEC and the run is whole.
template <typename T, int P, bool VEC>
__device__ __forceinline__ void load_chunk(const T *__restrict__ a, uint64_t p, uint64_t n, T (&out)[P])
{
    constexpr int B = P * (int)sizeof(T);
    if (VEC && p + P <= n) {
        if constexpr (B == 4) {
            const uint32_t w = *reinterpret_cast<const uint32_t *>(a + p);
            memcpy(&out[0], &w, 4);
        } else if constexpr (B == 8) {
            const uint2 w = *reinterpret_cast<const uint2 *>(a + p);
            memcpy(&out[0], &w, 8);
        } else {
            static_assert(B % 16 == 0, "chunk bytes");
            uint4 w[B / 16];
#pragma unroll
            for (int i = 0; i < B / 16; ++i) w[i] = reinterpret_cast<const uint4 *>(a + p)[i];
            memcpy(&out[0], &w[0], B);
        }
    } else {
#pragma unroll
        for (int j = 0; j < P; ++j) out[j] = p + j < n ? a[p + j] : T(0);
    }
}

template <typename T>
__device__ __forceinline__ T shfl_up_any(T v, int d)
{
    if constexpr (sizeof(T) == 8) return (T)__shfl_up_sync(0xFFFFFFFFu, (unsigned long long)v, d);
    else return (T)__shfl_up_sync(0xFFFFFFFFu, (uint32_t)v, d);
}

template <typename T>
__device__ __forceinline__ T shfl_any(T v, int src)
{
    if constexpr (sizeof(T) == 8) return (T)__shfl_sync(0xFFFFFFFFu, (unsigned long long)v, src);
    else return (T)__shfl_sync(0xFFFFFFFFu, (uint32_t)v, src);
}

// What the scan reads: sorted keys, the previous round's group ids, both, or
// precomputed boundary flags.
enum ScanMode { kScanKeys = 1, kScanGroup = 2, kScanKeysGroup = 3, kScanFlags = 4 };

// Position layout of a tile.  Warp w owns the 512 positions starting at
// tile base + w * 512, in C chunks of 32 * P; in chunk c lane l owns the P
// consecutive positions starting at c * 32 * P + l * P.  P is chosen so that
// a lane's run of the widest array read is 16 bytes: each warp load
// instruction then reads 512 contiguous bytes (whole sectors, each once).
template <typename K, int MODE>
struct ScanLayout {
    static constexpr bool kKeys = (MODE & kScanKeys) != 0;
    static constexpr bool kGroup = (MODE & kScanGroup) != 0;
    static constexpr bool kFlags = MODE == kScanFlags;
    static constexpr int kKeyBytes = kKeys ? (int)sizeof(K) : 1;
    static constexpr int kWidest = kFlags ? 1 : (kGroup && kKeyBytes < 4 ? 4 : kKeyBytes);
    static constexpr int P = 16 / kWidest;
    static constexpr int C = kScanItems / P;
    // per-chunk counts packed into one 64-bit word, in fields wide enough for
    // a warp's sum (at most 32 * P)
    static constexpr int FW = 32 * P <= 255 ? 8 : 16;
    static_assert(C * FW <= 64, "packed chunk counts");
};

// The boundary flags of one lane's rows: bit c * P + j is set when position
// wb + c * 32 * P + lane * P + j starts a group (its key or in_group differs
// from the previous position's, or it is position 0; or its flag is set).
// wb is the first position of the calling warp's 32 * kScanItems.  The whole
// warp calls it.
template <typename K, int MODE, bool VEC>
__device__ __forceinline__ uint32_t lane_flags(const K *__restrict__ keys, const uint32_t *__restrict__ in_group,
                                               const uint8_t *__restrict__ flags, uint64_t n, uint64_t wb, int lane)
{
    using L = ScanLayout<K, MODE>;
    constexpr int P = L::P, C = L::C;
    uint32_t fl = 0;
    if (wb >= n) return 0;   // warp-uniform
    K v[C][P];
    K vprev = K(0);        // lane 0: the key before the warp's first position
    uint32_t g[C][P];
    uint32_t gprev = 0;
    uint8_t f[C][P];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const uint64_t p = wb + (uint64_t)c * (32 * P) + (uint64_t)lane * P;
        if constexpr (L::kKeys) load_chunk<K, P, VEC>(keys, p, n, v[c]);
        if constexpr (L::kGroup) load_chunk<uint32_t, P, VEC>(in_group, p, n, g[c]);
        if constexpr (L::kFlags) load_chunk<uint8_t, P, VEC>(flags, p, n, f[c]);
    }
    if (lane == 0 && wb > 0) {
        if constexpr (L::kKeys) vprev = keys[wb - 1];
        if constexpr (L::kGroup) gprev = in_group[wb - 1];
    }
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const uint64_t p = wb + (uint64_t)c * (32 * P) + (uint64_t)lane * P;
        uint32_t bits = 0;
        if constexpr (L::kFlags) {
#pragma unroll
            for (int j = 0; j < P; ++j) bits |= (uint32_t)(f[c][j] != 0) << j;
        } else {
            if constexpr (L::kKeys) {
                // the item before each lane's run: the previous lane's last,
                // the last lane's of the previous chunk, or vprev
                const K up = shfl_up_any(v[c][P - 1], 1);
                const K wrap = c > 0 ? shfl_any(v[c > 0 ? c - 1 : 0][P - 1], 31) : vprev;
                K prev = lane == 0 ? wrap : up;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    bits |= (uint32_t)(v[c][j] != prev) << j;
                    prev = v[c][j];
                }
            }
            if constexpr (L::kGroup) {
                const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, g[c][P - 1], 1);
                const uint32_t wrap = c > 0 ? __shfl_sync(0xFFFFFFFFu, g[c > 0 ? c - 1 : 0][P - 1], 31) : gprev;
                uint32_t prev = lane == 0 ? wrap : up;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    bits |= (uint32_t)(g[c][j] != prev) << j;
                    prev = g[c][j];
                }
            }
            if (p == 0) bits |= 1u;
        }
        // positions past n
        if (p >= n) bits = 0;
        else if (n - p < (uint64_t)P) bits &= (1u << (uint32_t)(n - p)) - 1u;
        fl |= bits << (c * P);
    }
    return fl;
}

// Pass 1: the number of group starts in every tile of kScanTile positions
// (one block per tile; the keys stream through once).  With `masks`, each
// thread also stores its 16-bit boundary mask (2 bytes per 16 rows), so that
// pass 3 need not read the keys again.
template <typename K, int MODE, bool VEC>
__global__ void __launch_bounds__(kScanThreads, 2)
scan_count_kernel(const K *__restrict__ keys, const uint32_t *__restrict__ in_group, const uint8_t *__restrict__ flags,
                  uint64_t n, uint32_t *__restrict__ tile_count, uint16_t *__restrict__ masks)
{
    kernel_prologue();
    static_assert(kScanItems == 16, "one 16-bit mask per thread");
    __shared__ uint32_t s_warp[kScanWarps];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t wb = (uint64_t)blockIdx.x * kScanTile + (uint64_t)warp * (32 * kScanItems);
    const uint32_t fl = lane_flags<K, MODE, VEC>(keys, in_group, flags, n, wb, lane);
    if (masks) masks[(uint64_t)blockIdx.x * kScanThreads + threadIdx.x] = (uint16_t)fl;
    uint32_t c = __popc(fl);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane == 0) s_warp[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kScanWarps; ++w) t += s_warp[w];
        tile_count[blockIdx.x] = t;
    }
}

// Pass 2 (one block): exclusive prefix of the tile counts; the total is the
// group count, and (for segment extraction) the sentinel after the last
// segment start.
__global__ void __launch_bounds__(1024) scan_prefix_kernel(const uint32_t *__restrict__ tile_count, uint32_t tiles,
                                                           uint32_t *__restrict__ tile_prefix, uint32_t *d_count,
                                                           uint32_t *seg_start, uint64_t n)
{
    kernel_prologue();
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < tiles ? tile_count[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0u;
            uint32_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
                if (lane >= o) wi += y;
            }
            s_warp[lane] = wi - w;
        }
        __syncthreads();
        const uint32_t excl = s_carry + s_warp[warp] + incl - v;
        if (i < tiles) tile_prefix[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (d_count) *d_count = s_carry;
        if (seg_start) seg_start[s_carry] = (uint32_t)n;
    }
}

// Pass 3: the group ids (and segment starts) of every tile, from its prefix
// and the boundary masks of pass 1 (or, without them, the masks recomputed
// from the keys; tiles are then taken last first, since the keys that pass 1
// read last are the ones still in L2).
template <typename K, int MODE, bool VEC, bool MASKS>
__global__ void __launch_bounds__(kScanThreads, 2)
scan_ids_kernel(const K *__restrict__ keys, const uint32_t *__restrict__ in_group, const uint8_t *__restrict__ flags,
                uint64_t n, const uint32_t *__restrict__ tile_prefix, const uint16_t *__restrict__ masks,
                uint32_t *__restrict__ out_group, uint32_t *__restrict__ seg_start)
{
    kernel_prologue();
    using L = ScanLayout<K, MODE>;
    constexpr int P = L::P, C = L::C, FW = L::FW;
    constexpr uint32_t kChunkMask = (1u << P) - 1u;
    constexpr unsigned long long kFieldMask = (1ull << FW) - 1ull;
    __shared__ uint32_t s_warp[kScanWarps];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t tile = MASKS ? blockIdx.x : gridDim.x - 1 - blockIdx.x;
    const uint64_t wb = (uint64_t)tile * kScanTile + (uint64_t)warp * (32 * kScanItems);
    uint32_t fl;
    if constexpr (MASKS) fl = masks[(uint64_t)tile * kScanThreads + threadIdx.x];
    else fl = lane_flags<K, MODE, VEC>(keys, in_group, flags, n, wb, lane);
    // per chunk: the lane's exclusive count within the warp, packed
    unsigned long long wcnt = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) wcnt |= (unsigned long long)__popc((fl >> (c * P)) & kChunkMask) << (c * FW);
    unsigned long long incl = wcnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned long long tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const unsigned long long excl_l = incl - wcnt;
    if (lane == 31) {
        uint32_t wsum = 0;   // the warp's count
#pragma unroll
        for (int c = 0; c < C; ++c) wsum += (uint32_t)((tot >> (c * FW)) & kFieldMask);
        s_warp[warp] = wsum;
    }
    __syncthreads();
    // groups started before the warp: before the tile, in its earlier warps
    uint32_t first = tile_prefix[tile];
    for (int w = 0; w < warp; ++w) first += s_warp[w];
    if (wb >= n) return;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const uint64_t p = wb + (uint64_t)c * (32 * P) + (uint64_t)lane * P;
        // groups started before this lane's run in the chunk
        const uint32_t cfirst = first + (uint32_t)((excl_l >> (c * FW)) & kFieldMask);
        first += (uint32_t)((tot >> (c * FW)) & kFieldMask);
        if (p >= n) continue;
        const uint32_t bits = (fl >> (c * P)) & kChunkMask;
        if (out_group) {
            // 1-based id of the group holding position p + j, minus one
            uint32_t o[P];
            uint32_t id = cfirst;
#pragma unroll
            for (int j = 0; j < P; ++j) {
                id += (bits >> j) & 1u;
                o[j] = id - 1u;
            }
            if (VEC && p + P <= n) {
                if constexpr (P == 2) {
                    *reinterpret_cast<uint2 *>(out_group + p) = make_uint2(o[0], o[1]);
                } else {
#pragma unroll
                    for (int w = 0; w < P / 4; ++w)
                        reinterpret_cast<uint4 *>(out_group + p)[w] =
                            make_uint4(o[4 * w], o[4 * w + 1], o[4 * w + 2], o[4 * w + 3]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < P; ++j)
                    if (p + j < n) out_group[p + j] = o[j];
            }
        }
        if (seg_start) {
            uint32_t sid = cfirst;
            for (uint32_t m = bits; m; m &= m - 1) seg_start[sid++] = (uint32_t)(p + (__ffs(m) - 1));
        }
    }
}

template <typename K, int MODE, bool VEC>
void launch_scan_mode(cudaStream_t st, const K *keys, const uint32_t *in_group, const uint8_t *flags,
                      uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *tile_work, uint16_t *masks,
                      uint32_t *d_count)
{
    const uint32_t tiles = (uint32_t)((n + kScanTile - 1) / kScanTile);
    uint32_t *tile_count = tile_work, *tile_prefix = tile_work + tiles;
    launch_k(scan_count_kernel<K, MODE, VEC>, tiles, kScanThreads, 0, st, keys, in_group, flags, n, tile_count, masks);
    launch_k(scan_prefix_kernel, 1, 1024, 0, st, (const uint32_t *)tile_count, tiles, tile_prefix, d_count, seg_start, n);
    if (masks)
        launch_k(scan_ids_kernel<K, MODE, VEC, true>, tiles, kScanThreads, 0, st, keys, in_group, flags, n,
                 (const uint32_t *)tile_prefix, (const uint16_t *)masks, out_group, seg_start);
    else
        launch_k(scan_ids_kernel<K, MODE, VEC, false>, tiles, kScanThreads, 0, st, keys, in_group, flags, n,
                 (const uint32_t *)tile_prefix, (const uint16_t *)masks, out_group, seg_start);
}

// Launches the three passes for what the scan reads, with vector accesses
// when every array is 16-byte aligned.  tile_work holds 2 words per tile;
// masks (optional) kScanThreads 16-bit words per tile.
template <typename K>
void launch_scan(cudaStream_t st, const K *keys, const uint32_t *in_group, const uint8_t *flags,
                 uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *tile_work, uint16_t *masks,
                 uint32_t *d_count)
{
    const bool vec = (((uintptr_t)keys | (uintptr_t)in_group | (uintptr_t)flags | (uintptr_t)out_group) & 15u) == 0;
    const int mode = flags ? kScanFlags : (keys ? kScanKeys : 0) | (in_group ? kScanGroup : 0);
#define FMCS_SCAN_MODE(M)                                                                                        \
    (vec ? launch_scan_mode<K, M, true>(st, keys, in_group, flags, out_group, seg_start, n, tile_work, masks,    \
                                        d_count)                                                               \
         : launch_scan_mode<K, M, false>(st, keys, in_group, flags, out_group, seg_start, n, tile_work, masks,   \
                                         d_count))
    switch (mode) {
    case kScanKeys: FMCS_SCAN_MODE(kScanKeys); break;
    case kScanKeysGroup: FMCS_SCAN_MODE(kScanKeysGroup); break;
    case kScanFlags: FMCS_SCAN_MODE(kScanFlags); break;
    case kScanGroup: FMCS_SCAN_MODE(kScanGroup); break;
    default: FMCS_SCAN_MODE(0); break;   // nothing to compare: one group
    }
#undef FMCS_SCAN_MODE
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
    if (tiles > 0xFFFFFFFFull) return set_error(ctx, FMCS_E_INVAL, "boundary scan: too many rows");
    void *tw = nullptr;
    int rc = ws_get(ctx, kSlotScanTiles,
                    carve_total({tiles * 2 * sizeof(uint32_t), tiles * kScanThreads * sizeof(uint16_t)}), &tw);
    if (rc) return rc;
    Carver cv(tw);
    uint32_t *tile_work = cv.take<uint32_t>(2 * tiles);   // per tile: group-start count, then prefix
    uint16_t *masks = cv.take<uint16_t>(tiles * kScanThreads);   // per thread of every tile: its boundary mask
    LaunchScope ls_(ctx, "boundary_scan");
    switch (keys ? key_bytes : 0) {
    case 0:
        launch_scan<uint32_t>(ctx->stream, nullptr, in_group, flags, out_group, seg_start, n, tile_work, masks,
                              d_count);
        break;
    case 1:
        launch_scan<uint8_t>(ctx->stream, (const uint8_t *)keys, in_group, flags, out_group, seg_start, n, tile_work,
                             masks, d_count);
        break;
    case 2:
        launch_scan<uint16_t>(ctx->stream, (const uint16_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_work, masks, d_count);
        break;
    case 4:
        launch_scan<uint32_t>(ctx->stream, (const uint32_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_work, masks, d_count);
        break;
    case 8:
        launch_scan<uint64_t>(ctx->stream, (const uint64_t *)keys, in_group, flags, out_group, seg_start, n,
                              tile_work, masks, d_count);
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
// imply.  fmcs_group_ids_noalloc serves them: the same boundary scan as the
// group ids of a sort round, with its scratch (the per-tile group-start counts
// and their prefixes, and the group count) in the file-scope device array
// below instead of the context's workspace.  The caller passes device inputs
// and outputs on the current device; no context is needed.
//
// The array is modest (kNoAllocTiles 64-bit words, 128 KiB) and every GPU
// that loads the library holds it until the process exits.  n is bounded at
// 67,108,864 rows (at most 8,192 scan tiles).  All calls share it and it keeps the
// last call's contents, so each call clears the word that must start at zero
// (the group count; the counts and prefixes are written before they are read);
// calls whose work overlaps on the GPU (two streams, or two host threads)
// race on it and must be serialized by the caller.  The scan's three passes
// have no waits between blocks, so the call has no timeout path.
//
// The call is synchronous: it waits for its stream before it returns the
// group count.  Its first call on a device resolves the array's device address
// (cudaGetSymbolAddress, once per device, with that device current); make that
// first call before any stream capture begins on the device.
// ---------------------------------------------------------------------------
namespace fmcs {
namespace {

constexpr uint64_t kNoAllocTiles = 16384;
constexpr uint64_t kNoAllocMaxRows = 67108864;
static_assert(kNoAllocMaxRows / kScanTile <= kNoAllocTiles, "a count and a prefix word for every tile");
// layout (64-bit words): [0, kNoAllocTiles) the tiles' counts and prefixes
// (two 32-bit words per tile); then a spare word and the group count, one
// 64-bit word each
constexpr uint64_t kNoAllocWords = kNoAllocTiles + 2;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long *g_noalloc_ptr[kMaxDevices] = {};

// True when p is device (or managed) memory that the current device can use
// as its own: device memory of another GPU is refused.
bool on_current_device(const void *p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (attr.type == cudaMemoryTypeManaged) return true;
    if (attr.type != cudaMemoryTypeDevice) return false;
    int dev = -1;
    return cudaGetDevice(&dev) == cudaSuccess && attr.device == dev;
}

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
    // device pointers of the current device only: staging host data would
    // allocate, and the scratch and the launches belong to the current device
    if (!keys || !out_group || !on_current_device(keys) || !on_current_device(out_group) ||
        (in_group && !on_current_device(in_group)))
        return FMCS_E_INVAL;
    unsigned long long *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *tile_work = (uint32_t *)scratch;   // per tile: group-start count, then prefix
    uint32_t *d_count = (uint32_t *)(scratch + kNoAllocTiles + 1);
    // the previous call's group count starts at zero
    cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return FMCS_E_CUDA;
    switch (key_bytes) {
    case 1:
        launch_scan<uint8_t>(st, (const uint8_t *)keys, in_group, nullptr, out_group, nullptr, n, tile_work, nullptr,
                             d_count);
        break;
    case 2:
        launch_scan<uint16_t>(st, (const uint16_t *)keys, in_group, nullptr, out_group, nullptr, n, tile_work,
                              nullptr, d_count);
        break;
    case 4:
        launch_scan<uint32_t>(st, (const uint32_t *)keys, in_group, nullptr, out_group, nullptr, n, tile_work,
                              nullptr, d_count);
        break;
    default:
        launch_scan<uint64_t>(st, (const uint64_t *)keys, in_group, nullptr, out_group, nullptr, n, tile_work,
                              nullptr, d_count);
        break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return FMCS_E_CUDA;
    // read the count back (into the caller's stack: no allocation) and finish
    // the call
    uint32_t back = 0;
    e = cudaMemcpyAsync(&back, d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return FMCS_E_CUDA;
    if (ngroups) *ngroups = back;
    return FMCS_OK;
}
