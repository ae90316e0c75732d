// fmcs_internal.h -- host-side internals of libfmcs: the context (stream,
// device workspace, status word), the workspace slots, and the launchers of
// the sm_100a kernels.  Not part of the public ABI (include/fmcs_capi.h).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <functional>
#include <initializer_list>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fmcs_capi.h"

namespace fmcs {

// Named workspace slots; each grows on demand and is reused across calls.
enum Slot : int {
    kSlotKeys0 = 0,   // sort engine buffer 0 keys (final when the caller wants no keys)
    kSlotKeys1,       // sort engine buffer 1 keys
    kSlotVals1,       // sort engine buffer 1 vals
    kSlotVals0,       // sort engine buffer 0 vals when the caller's order is host memory
    kSlotSegStart,    // initial segment starts (n + 2)
    kSlotLarge0,      // large-segment descriptors, ping
    kSlotLarge1,      // large-segment descriptors, pong
    kSlotSegHist,     // per large segment digit histograms / offsets
    kSlotTilePrefix,  // tile prefix per large segment
    kSlotLookback,    // look-back words
    kSlotLocalA,      // local lists, warp tier
    kSlotLocalB,      // block tier (medium)
    kSlotLocalC,      // block tier (large)
    kSlotCounters,    // small device counters
    kSlotScanTiles,   // look-back words of the flag scans
    kSlotHashTable,   // hash grouping table
    kSlotHashIdx,     // hash grouping per-row ids
    kSlotStageIn0,    // host-staging buffers
    kSlotStageIn1,
    kSlotStageIn2,
    kSlotStageOut0,
    kSlotStageOut1,
    kSlotStageOut2,
    kSlotBank0,       // run_plan banks
    kSlotBank1,
    kSlotBank2,
    kSlotBank3,
    kSlotGroupA,      // run_plan group ping
    kSlotGroupB,      // run_plan group pong
    kSlotColStage,    // run_plan host column staging (several columns)
    kSlotTopHist,     // level-0 digit histogram of a round-0 bank, counted by the stitch
    kSlotMisc,
    kSlotCount
};

struct Workspace {
    void *ptr[kSlotCount] = {};
    size_t cap[kSlotCount] = {};
};

}  // namespace fmcs

struct fmcs_prof_rec {
    const char *name;
    cudaEvent_t a, b;
    double units;   // work items of the launch (rows), when the launcher knows them
    double bytes;   // algorithmic HBM bytes of the launch, when the launcher knows them
    int round;      // sort/hash round of a plan the launch belongs to (-1: none)
};

struct fmcs_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;     // capture stream of conditional-node bodies (created on first use)
    // a second stream for independent work of one call (the on-chip tiers
    // split in two groups) and its fork / join events (created on first use)
    cudaStream_t par = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    size_t budget = 0;   // 0 = unlimited
    size_t held = 0;     // bytes held by the workspace
    fmcs::Workspace ws;
    int *d_status = nullptr;       // device status word
    uint32_t epoch = 1;            // look-back epoch, advanced per launch
    std::string err;
    int *h_status = nullptr;       // pinned mirror of the status word
    uint32_t *h_small = nullptr;   // pinned small read-back area (64 words)
    // kernel profiler: CUDA events around every launch while enabled
    bool prof_on = false;
    std::vector<fmcs_prof_rec> prof;
    std::vector<cudaEvent_t> ev_pool;
    unsigned long long launches = 0;   // kernels launched by this context
    cudaEvent_t ev_level = nullptr;    // host-side read-back point of the sort levels
    // tuned knobs (the autotuner's tuning/b200.json, FMCS_TUNING, or fmcs_set_tuning)
    int rank_mode = 0;                 // 0: match.any multi-split, 1: ballot, 2: shared-memory OR
    uint32_t local_max = 8192;         // segments above this many rows take the MSD levels
    uint32_t msd_items = 8;            // items per thread of an MSD tile (8 or 16)
    int prof_round = -1;               // round tag of the launches being profiled
};

namespace fmcs {

// Sub-arrays carved out of one workspace slot.  Each starts on a
// kCarveAlign-byte boundary (a slot comes from cudaMalloc, so its base is
// 256-byte aligned), whatever the sizes of the sub-arrays before it: a kernel
// may read any of them with 16-byte vectors.
constexpr size_t kCarveAlign = 256;
inline size_t carve_round(size_t bytes) { return (bytes + kCarveAlign - 1) & ~(kCarveAlign - 1); }
// Bytes of a slot that holds sub-arrays of these sizes in bytes.
inline size_t carve_total(std::initializer_list<size_t> sizes)
{
    size_t t = 0;
    for (size_t b : sizes) t += carve_round(b);
    return t;
}
class Carver {
  public:
    explicit Carver(void *base) : cur_(static_cast<char *>(base)) {}
    template <typename T>
    T *take(size_t count)
    {
        T *p = reinterpret_cast<T *>(cur_);
        cur_ += carve_round(count * sizeof(T));
        return p;
    }

  private:
    char *cur_;
};

int set_error(fmcs_ctx *ctx, int code, const std::string &msg);
int cuda_fail(fmcs_ctx *ctx, cudaError_t e, const char *what);
// Returns a device pointer of at least `bytes` in `slot` (grown as needed).
int ws_get(fmcs_ctx *ctx, int slot, size_t bytes, void **out, bool zero_new = false);
// Checks and clears the device status word (synchronizes the stream).
int check_status(fmcs_ctx *ctx, const char *what);

// Brackets one kernel launch: counts it and, while profiling is on, records
// a pair of CUDA events on the context's stream around it.
class LaunchScope {
  public:
    LaunchScope(fmcs_ctx *ctx, const char *name);
    ~LaunchScope();
    void set_units(double u);
    void set_bytes(double b);

  private:
    fmcs_ctx *ctx_;
    int rec_ = -1;
};

// Appends a WHILE conditional node to the graph being captured on `st` and
// captures body(stream, handle) as the loop body.  The handle is 1 at the
// start of every graph launch; a kernel of the body sets it to 0 (with
// cudaGraphSetConditional) to end the loop.
int capture_while(fmcs_ctx *ctx, cudaStream_t st,
                  const std::function<int(cudaStream_t, cudaGraphConditionalHandle)> &body);

// The context's second stream and its fork/join events (created on first
// use): fork makes `par` wait for the work enqueued on `st` so far, join makes
// `st` wait for the work enqueued on `par`.
int par_stream(fmcs_ctx *ctx, cudaStream_t *par);
int fork_par(fmcs_ctx *ctx, cudaStream_t st);
int join_par(fmcs_ctx *ctx, cudaStream_t st);

// Launches a library kernel with programmatic stream serialization: it may
// begin launching while the stream's previous kernel finishes (its prologue
// waits for that kernel's completion).  Every kernel launched this way starts
// with kernel_prologue().
template <typename... P, typename... A>
inline cudaError_t launch_k(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A &&...args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// True when the device can dereference p directly (device or managed memory).
bool is_device_ptr(const void *p);

// ---------------------------------------------------------------- stitch
struct StitchSlice {
    const void *src;
    uint32_t src_bytes;
    uint32_t rshift;   // src_bits - end
    uint32_t width;    // end - start + 1
    uint32_t invert;   // 1: the slice's bits are inverted (its column sorts descending)
};
constexpr int kMaxSlices = 32;
// With top_hist (device, 256 words per chunk of chunk_rows rows and one more
// row), the stitch also counts the top digit (bits [key_bits - min(8,
// key_bits), key_bits)) of every bank value, one row per chunk and the total
// in the last row: the first radix level's histograms of a round-0 sort of
// the bank (chunk_rows = msd_chunk_rows).
// `stream`: NULL for the context's stream.
int launch_stitch(fmcs_ctx *ctx, const StitchSlice *sl, int ns, void *bank, uint32_t bank_bytes,
                  uint64_t n, uint32_t *top_hist = nullptr, uint32_t key_bits = 0, uint32_t chunk_rows = 0,
                  cudaStream_t stream = nullptr);

// bank[i] <<= lshift (src == NULL) or bank[i] |= (src[i] >> rshift) & mask(width)
int launch_bank_update(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n, uint32_t lshift,
                       const void *src, uint32_t src_bytes, uint32_t rshift, uint32_t width);

// ---------------------------------------------------------------- gather
int launch_gather(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, const uint32_t *order,
                  void *out, uint64_t n);

// ---------------------------------------------------------------- sort engine
struct SortArgs {
    const void *bank;          // device, bank_bytes per row (row order)
    uint32_t bank_bytes;       // 2, 4 or 8
    uint32_t key_bits;         // significant bits
    const uint32_t *order_in;  // device, NULL for round 0 (iota)
    const uint32_t *seg_start; // device, nseg+1 entries (seg_start[nseg] == n), or NULL = one segment
    uint32_t nseg_host;        // nseg when known on the host (seg_start != NULL requires d_nseg)
    const uint32_t *d_nseg;    // device count of segments (with seg_start)
    uint32_t *order_out;       // device, n (may alias order_in)
    void *keys_out;            // device, n keys, or NULL
    uint64_t n;
    bool fixed_launches = false;  // launch every level (no host read-back), e.g. under graph capture
    const uint32_t *top_hist = nullptr;  // round 0 only: the first level's per-chunk digit histograms, already counted
    // Device-side overrides read by the round's first kernel (no host
    // read-back): the significant key bits (<= key_bits, which then only
    // bounds the number of radix levels), and a flag that, when non-zero,
    // says the rows are in order already (every segment is only copied).
    const uint32_t *d_key_bits = nullptr;
    const uint32_t *d_in_order = nullptr;
};
int sort_segments(fmcs_ctx *ctx, const SortArgs &a);
// Rows per look-back chunk of an HBM radix level (kChunkTiles tiles of the
// context's tile size): the row granularity of the per-chunk histograms.
uint32_t msd_chunk_rows(const fmcs_ctx *ctx);
// Stable full-array LSD radix sort of (keys, vals) in place by key bits
// [0, bits): the plain, unsegmented comparator path.
int lsd_sort_full(fmcs_ctx *ctx, void *keys, uint32_t key_bytes, uint32_t *vals, uint64_t n, uint32_t bits);

// ---------------------------------------------------------------- group ids / segments
// out_group[i] = number of boundaries in (0, i], boundary at i when
// keys[i] != keys[i-1] or (in_group && in_group[i] != in_group[i-1]).
// Optionally writes the group count to *d_ngroups (device) .
int launch_group_ids(fmcs_ctx *ctx, const void *keys, uint32_t key_bytes, const uint32_t *in_group,
                     uint32_t *out_group, uint64_t n, uint32_t *d_ngroups);
// seg_start[k] = position of the k-th run start of in_group; seg_start[S] = n;
// *d_nseg = S (device).
int launch_segments(fmcs_ctx *ctx, const uint32_t *in_group, uint32_t *seg_start, uint32_t *d_nseg,
                    uint64_t n);

// Group ids and, when seg_start != NULL, the start of every group (the next
// round's segments); *d_count = number of groups.
int launch_group_ids_segments(fmcs_ctx *ctx, const void *keys, uint32_t key_bytes, const uint32_t *in_group,
                              uint32_t *out_group, uint32_t *seg_start, uint64_t n, uint32_t *d_count);
// v[i] = i
int launch_iota(fmcs_ctx *ctx, uint32_t *v, uint64_t n);
// rank[i] = (number of set flags in [0, i]) - 1; *d_count = number of set flags.
int launch_flag_rank(fmcs_ctx *ctx, const uint8_t *flags, uint32_t *rank, uint64_t n, uint32_t *d_count);

// ---------------------------------------------------------------- hash grouping
// fixed_launches: the same launches whatever the data, with no host
// read-back (graph capture).
// Rows a hash round takes at most (less one): its table's slot indices are
// 32-bit words below two sentinels, so it holds at most 2^31 slots.
constexpr uint64_t kHashMaxRows = 1ull << 31;
int hash_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, const uint32_t *order_in,
               uint32_t *order_out, const uint32_t *in_group, uint32_t *out_group, uint64_t n,
               bool last_round, uint32_t *d_ngroups, bool group_is_key = false, bool fixed_launches = false);

}  // namespace fmcs
