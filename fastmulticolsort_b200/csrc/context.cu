// context.cu -- fmcs_ctx lifetime, the device workspace (named slots that grow
// on demand and are reused across calls; the reference instead mallocs and
// frees every buffer per call, src/common.h:18-31), the device status word that
// bounded waits report through, and error strings.
#include "device_common.cuh"
#include "fmcs_internal.h"

#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <cstring>

namespace fmcs {

int set_error(fmcs_ctx *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(fmcs_ctx *ctx, cudaError_t e, const char *what)
{
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return set_error(ctx, e == cudaErrorMemoryAllocation ? FMCS_E_OOM : FMCS_E_CUDA, buf);
}

int ws_get(fmcs_ctx *ctx, int slot, size_t bytes, void **out, bool zero_new)
{
    Workspace &w = ctx->ws;
    if (bytes == 0) bytes = 256;
    if (w.cap[slot] >= bytes) {
        *out = w.ptr[slot];
        return FMCS_OK;
    }
    size_t want = bytes + bytes / 8;
    want = (want + 4095) & ~size_t(4095);
    if (ctx->budget && ctx->held - w.cap[slot] + want > ctx->budget) {
        want = bytes;
        if (ctx->held - w.cap[slot] + want > ctx->budget) {
            char buf[200];
            snprintf(buf, sizeof(buf), "workspace budget exceeded: need %zu more bytes over %zu",
                     want, ctx->budget);
            return set_error(ctx, FMCS_E_OOM, buf);
        }
    }
    if (w.ptr[slot]) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "workspace sync");
        cudaFree(w.ptr[slot]);
        ctx->held -= w.cap[slot];
        w.ptr[slot] = nullptr;
        w.cap[slot] = 0;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(ctx, e, "workspace cudaMalloc");
    }
    if (zero_new) {
        // look-back words must not carry a stale (epoch, flag) from whatever
        // the allocation held before
        e = cudaMemsetAsync(p, 0, want, ctx->stream);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_fail(ctx, e, "workspace memset");
        }
    }
    w.ptr[slot] = p;
    w.cap[slot] = want;
    ctx->held += want;
    *out = p;
    return FMCS_OK;
}

int par_stream(fmcs_ctx *ctx, cudaStream_t *par)
{
    cudaError_t e = cudaSuccess;
    if (!ctx->par) e = cudaStreamCreateWithFlags(&ctx->par, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->ev_fork) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->ev_join) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "second stream");
    *par = ctx->par;
    return FMCS_OK;
}

int fork_par(fmcs_ctx *ctx, cudaStream_t st)
{
    cudaStream_t par = nullptr;
    int rc = par_stream(ctx, &par);
    if (rc) return rc;
    cudaError_t e = cudaEventRecord(ctx->ev_fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(par, ctx->ev_fork, 0);
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "fork");
}

int join_par(fmcs_ctx *ctx, cudaStream_t st)
{
    cudaError_t e = cudaEventRecord(ctx->ev_join, ctx->par);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ctx->ev_join, 0);
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "join");
}

int capture_while(fmcs_ctx *ctx, cudaStream_t st,
                  const std::function<int(cudaStream_t, cudaGraphConditionalHandle)> &body)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: capture info");
    if (cs != cudaStreamCaptureStatusActive) return set_error(ctx, FMCS_E_INVAL, "capture_while: stream not capturing");
    if (!ctx->side) {
        e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: stream");
    }
    cudaGraphConditionalHandle h;
    e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: handle");
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, ndeps, &np);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: node");
    cudaGraph_t bodyg = np.conditional.phGraph_out[0];
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: dependencies");
    e = cudaStreamBeginCaptureToGraph(ctx->side, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: body capture");
    cudaStream_t saved = ctx->stream;
    ctx->stream = ctx->side;
    int rc = body(ctx->side, h);
    ctx->stream = saved;
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(ctx->side, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture_while: body end");
    return FMCS_OK;
}

int check_status(fmcs_ctx *ctx, const char *what)
{
    cudaError_t e = cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    int s = *ctx->h_status;
    if (s != 0) {
        *ctx->h_status = 0;
        cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
        char buf[200];
        if (s == FMCS_E_TIMEOUT)
            snprintf(buf, sizeof(buf), "%s: a device-side wait timed out", what);
        else
            snprintf(buf, sizeof(buf), "%s: device reported status %d", what, s);
        return set_error(ctx, s == FMCS_E_TIMEOUT ? FMCS_E_TIMEOUT : FMCS_E_INVAL, buf);
    }
    return FMCS_OK;
}

static cudaEvent_t take_event(fmcs_ctx *ctx)
{
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

LaunchScope::LaunchScope(fmcs_ctx *ctx, const char *name) : ctx_(ctx)
{
    ctx->launches++;
    if (!ctx->prof_on) return;
    fmcs_prof_rec r{name, take_event(ctx), take_event(ctx), 0.0, 0.0, ctx->prof_round};
    if (!r.a || !r.b) return;
    cudaEventRecord(r.a, ctx->stream);
    rec_ = (int)ctx->prof.size();
    ctx->prof.push_back(r);
}

void LaunchScope::set_units(double u)
{
    if (rec_ >= 0) ctx_->prof[rec_].units = u;
}

void LaunchScope::set_bytes(double b)
{
    if (rec_ >= 0) ctx_->prof[rec_].bytes = b;
}

LaunchScope::~LaunchScope()
{
    if (rec_ >= 0) cudaEventRecord(ctx_->prof[rec_].b, ctx_->stream);
}

bool is_device_ptr(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Knobs of the autotuner's JSON (tuning/b200.json next to the library, or the
// file FMCS_TUNING names): "rank_mode", "local_max", "msd_items".
static bool json_number(const std::string &txt, const char *key, double *out)
{
    const std::string pat = std::string("\"") + key + "\"";
    size_t p = txt.find(pat);
    if (p == std::string::npos) return false;
    p = txt.find(':', p);
    if (p == std::string::npos) return false;
    char *end = nullptr;
    const double v = strtod(txt.c_str() + p + 1, &end);
    if (end == txt.c_str() + p + 1) return false;
    *out = v;
    return true;
}

static void load_tuning(fmcs_ctx *ctx)
{
    std::string path;
    if (const char *env = getenv("FMCS_TUNING")) {
        path = env;
    } else {
        Dl_info info;
        if (dladdr((void *)&load_tuning, &info) && info.dli_fname) {
            std::string f = info.dli_fname;
            size_t sl = f.rfind('/');
            path = (sl == std::string::npos ? std::string(".") : f.substr(0, sl)) + "/tuning/b200.json";
        }
    }
    std::ifstream f(path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string txt = ss.str();
    double v;
    if (json_number(txt, "rank_mode", &v) && v >= 0 && v <= 2) ctx->rank_mode = (int)v;
    if (json_number(txt, "local_max", &v) && v >= 128 && v <= 8192) ctx->local_max = (uint32_t)v;
    if (json_number(txt, "msd_items", &v)) ctx->msd_items = v >= 16 ? 16 : 8;
}

}  // namespace fmcs

using namespace fmcs;

extern "C" int fmcs_create(fmcs_ctx **out, int device, size_t hbm_budget_bytes)
{
    if (!out) return FMCS_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FMCS_E_CUDA;
    }
    if (device < 0 || device >= ndev) return FMCS_E_INVAL;
    fmcs_ctx *ctx = new fmcs_ctx();
    ctx->device = device;
    ctx->budget = hbm_budget_bytes;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, 256);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, 256);
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_small, 64 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_level, cudaEventDisableTiming);
    // the second stream and its events exist from the start, so that a call
    // made while the caller captures the context's stream creates nothing
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->par, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fmcs_destroy(ctx);
        return FMCS_E_CUDA;
    }
    *ctx->h_status = 0;
    load_tuning(ctx);
    if (const char *m = getenv("FMCS_RANK_MODE"))
        ctx->rank_mode = (m[0] == 'b' || m[0] == '1') ? 1 : (m[0] == 'o' || m[0] == '2') ? 2 : 0;
    *out = ctx;
    return FMCS_OK;
}

extern "C" void fmcs_destroy(fmcs_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int s = 0; s < kSlotCount; ++s)
        if (ctx->ws.ptr[s]) cudaFree(ctx->ws.ptr[s]);
    for (auto &r : ctx->prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_small) cudaFreeHost(ctx->h_small);
    if (ctx->ev_level) cudaEventDestroy(ctx->ev_level);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->par) cudaStreamDestroy(ctx->par);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char *fmcs_last_error(const fmcs_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int fmcs_synchronize(fmcs_ctx *ctx)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_synchronize");
    return FMCS_OK;
}

extern "C" void *fmcs_stream(fmcs_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" size_t fmcs_workspace_bytes(const fmcs_ctx *ctx) { return ctx ? ctx->held : 0; }

extern "C" int fmcs_profile(fmcs_ctx *ctx, int enable)
{
    if (!ctx) return FMCS_E_INVAL;
    ctx->prof_on = enable != 0;
    return FMCS_OK;
}

extern "C" unsigned long long fmcs_launch_count(const fmcs_ctx *ctx) { return ctx ? ctx->launches : 0; }

extern "C" int fmcs_profile_report(fmcs_ctx *ctx, char *buf, size_t len)
{
    if (!ctx || !buf || len == 0) return FMCS_E_INVAL;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_profile_report");
    struct Agg {
        std::string name;
        unsigned long long n = 0;
        double ms = 0;
        double units = 0;
        double bytes = 0;
    };
    std::vector<Agg> agg;
    std::vector<double> round_ms;
    for (auto &r : ctx->prof) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            ms = 0;
        }
        size_t k = 0;
        while (k < agg.size() && agg[k].name != r.name) ++k;
        if (k == agg.size()) agg.push_back(Agg{r.name});
        agg[k].n++;
        agg[k].ms += ms;
        agg[k].units += r.units;
        agg[k].bytes += r.bytes;
        // per-round totals of the sort/hash work (the stitch is reported apart)
        if (r.round >= 0 && strcmp(r.name, "stitch") != 0) {
            if ((int)round_ms.size() <= r.round) round_ms.resize(r.round + 1, 0.0);
            round_ms[r.round] += ms;
        }
        ctx->ev_pool.push_back(r.a);
        ctx->ev_pool.push_back(r.b);
    }
    ctx->prof.clear();
    std::string out = "{";
    for (size_t k = 0; k < agg.size(); ++k) {
        char tmp[256];
        snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %llu, \"ms\": %.6f, \"units\": %.0f, \"bytes\": %.0f}",
                 k ? ", " : "", agg[k].name.c_str(), agg[k].n, agg[k].ms, agg[k].units, agg[k].bytes);
        out += tmp;
    }
    if (!round_ms.empty()) {
        out += agg.empty() ? "\"_round_ms\": [" : ", \"_round_ms\": [";
        for (size_t r = 0; r < round_ms.size(); ++r) {
            char tmp[64];
            snprintf(tmp, sizeof(tmp), "%s%.6f", r ? ", " : "", round_ms[r]);
            out += tmp;
        }
        out += "]";
    }
    out += "}";
    if (out.size() + 1 > len) return set_error(ctx, FMCS_E_INVAL, "fmcs_profile_report: buffer too small");
    memcpy(buf, out.c_str(), out.size() + 1);
    return FMCS_OK;
}

extern "C" int fmcs_set_tuning(fmcs_ctx *ctx, const char *key, long long value)
{
    if (!ctx || !key) return FMCS_E_INVAL;
    const std::string k(key);
    if (k == "rank_mode") {
        if (value < 0 || value > 2) return set_error(ctx, FMCS_E_INVAL, "rank_mode must be 0, 1 or 2");
        ctx->rank_mode = (int)value;
    } else if (k == "local_max") {
        if (value < 128 || value > 8192) return set_error(ctx, FMCS_E_INVAL, "local_max must be in 128..8192");
        ctx->local_max = (uint32_t)value;
    } else if (k == "msd_items") {
        if (value != 8 && value != 16) return set_error(ctx, FMCS_E_INVAL, "msd_items must be 8 or 16");
        ctx->msd_items = (uint32_t)value;
    } else {
        return set_error(ctx, FMCS_E_INVAL, "unknown tuning key " + k);
    }
    return FMCS_OK;
}

extern "C" long long fmcs_get_tuning(const fmcs_ctx *ctx, const char *key)
{
    if (!ctx || !key) return -1;
    const std::string k(key);
    if (k == "rank_mode") return ctx->rank_mode;
    if (k == "local_max") return ctx->local_max;
    if (k == "msd_items") return ctx->msd_items;
    return -1;
}

// ---------------------------------------------------------------------------
// Self-test of the bounded device waits: one warp waits, through lb_wait (the
// wait every look-back of the library uses), on a word of the workspace that
// no kernel writes.  The wait must give up after `polls` polls, record
// FMCS_E_TIMEOUT in the context's status word and return, leaving the
// context usable.
// ---------------------------------------------------------------------------
namespace fmcs {
namespace {
__global__ void selftest_wait_kernel(const unsigned long long *word, uint32_t epoch, int *status, uint32_t polls,
                                     uint32_t *out)
{
    kernel_prologue();
    const unsigned long long w = lb_wait(word, epoch, status, polls);
    if (threadIdx.x == 0) *out = (uint32_t)w;
}
}  // namespace
}  // namespace fmcs

extern "C" int fmcs_selftest_wait(fmcs_ctx *ctx, uint32_t polls)
{
    using namespace fmcs;
    if (!ctx) return FMCS_E_INVAL;
    if (polls < 1 || polls > (1u << 20)) return set_error(ctx, FMCS_E_INVAL, "polls must be in 1..2^20");
    void *p = nullptr;
    int rc = ws_get(ctx, kSlotMisc, 256, &p);
    if (rc) return rc;
    // a zero word carries epoch 0 and no flag: a wait for epoch 1 never ends
    // on it, and nothing else writes the word while this call runs
    cudaError_t e = cudaMemsetAsync(p, 0, 256, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "selftest memset");
    {
        LaunchScope ls_(ctx, "selftest_wait");
        launch_k(selftest_wait_kernel, 1, 32, 0, ctx->stream, (const unsigned long long *)p, 1u, ctx->d_status,
                 polls, (uint32_t *)p + 16);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "selftest launch");
    return check_status(ctx, "fmcs_selftest_wait");
}
