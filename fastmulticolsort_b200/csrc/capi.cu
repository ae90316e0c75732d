// capi.cu -- the extern "C" entry points of include/fmcs_capi.h.
//
// Host-side orchestration of one round / one plan: argument checks (the
// reference asserts or exits instead, e.g. src/mergesort.h:2926-2931,
// src/stitch_composer.cpp:684-687), host<->device staging for host pointers,
// the round loop of Composer::multiRoundSorting (src/composer.cpp:48-135) and
// of StitchComposer::run_single_plan (src/stitch_composer.cpp:555-806), and the
// final status check of the bounded device waits.
#include "device_common.cuh"
#include "fmcs_internal.h"
#include "plan.h"

#include <cstring>
#include <vector>

namespace fmcs {

namespace {

constexpr int kCtrNgroups = 40;   // counters slot word for group counts

// Device view of an input: the pointer itself, or a staged copy of host data.
int stage_in(fmcs_ctx *ctx, const void *p, size_t bytes, int slot, const void **out)
{
    if (!p) {
        *out = nullptr;
        return FMCS_OK;
    }
    if (is_device_ptr(p)) {
        *out = p;
        return FMCS_OK;
    }
    void *d;
    int rc = ws_get(ctx, slot, bytes, &d);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stage in");
    *out = d;
    return FMCS_OK;
}

// Device view of an output: the pointer itself, or a staging buffer that is
// copied back by copy_out.
int stage_out(fmcs_ctx *ctx, void *p, size_t bytes, int slot, void **out, bool *host)
{
    *host = false;
    if (!p) {
        *out = nullptr;
        return FMCS_OK;
    }
    if (is_device_ptr(p)) {
        *out = p;
        return FMCS_OK;
    }
    *host = true;
    return ws_get(ctx, slot, bytes, out);
}

int copy_out(fmcs_ctx *ctx, void *host, const void *dev, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    return e == cudaSuccess ? FMCS_OK : cuda_fail(ctx, e, "copy out");
}

bool valid_bank(uint32_t b) { return b == 1 || b == 2 || b == 4 || b == 8; }

int finish(fmcs_ctx *ctx, const char *what, uint32_t *ngroups, const uint32_t *d_ng)
{
    if (ngroups && d_ng) {
        cudaError_t e = cudaMemcpyAsync(ctx->h_small + 1, d_ng, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    }
    int rc = check_status(ctx, what);   // synchronizes
    if (rc) return rc;
    if (ngroups) *ngroups = d_ng ? ctx->h_small[1] : 0;
    return FMCS_OK;
}

int counters(fmcs_ctx *ctx, uint32_t **w)
{
    void *p;
    int rc = ws_get(ctx, kSlotCounters, 4096, &p);
    *w = (uint32_t *)p;
    return rc;
}

// One sort round on device data.  order (device) is in/out; seg_start/d_nseg
// describe the runs of in_group when the caller already has them.
int sort_round_dev(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t key_bits, uint32_t *order,
                   const uint32_t *in_group, const uint32_t *seg_start, const uint32_t *d_nseg,
                   uint32_t *out_group, void *keys_out, uint32_t *next_seg_start, uint32_t *d_next_nseg,
                   uint64_t n, uint32_t *d_ngroups, bool identity_order = false, bool fixed_launches = false,
                   const uint32_t *top_hist = nullptr)
{
    int rc;
    void *p;
    if (!keys_out) {
        if ((rc = ws_get(ctx, kSlotKeys0, n * bank_bytes, &p))) return rc;
        keys_out = p;
    }
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    if (in_group && !seg_start) {
        if ((rc = ws_get(ctx, kSlotSegStart, (n + 2) * sizeof(uint32_t), &p))) return rc;
        uint32_t *ss = (uint32_t *)p;
        if ((rc = launch_segments(ctx, in_group, ss, w + kCtrNgroups + 1, n))) return rc;
        seg_start = ss;
        d_nseg = w + kCtrNgroups + 1;
    }
    SortArgs a;
    a.bank = bank;
    a.bank_bytes = bank_bytes;
    a.key_bits = key_bits;
    a.order_in = (in_group && !identity_order) ? order : nullptr;
    a.seg_start = in_group ? seg_start : nullptr;
    a.nseg_host = 0;
    a.d_nseg = in_group ? d_nseg : nullptr;
    a.order_out = order;
    a.keys_out = keys_out;
    a.n = n;
    a.fixed_launches = fixed_launches;
    a.top_hist = in_group ? nullptr : top_hist;
    if ((rc = sort_segments(ctx, a))) return rc;
    if (out_group || next_seg_start)
        return launch_group_ids_segments(ctx, keys_out, bank_bytes, in_group, out_group, next_seg_start, n,
                                         next_seg_start ? d_next_nseg : d_ngroups);
    return FMCS_OK;
}

// The device work of one plan (stitch + rounds), enqueued on the context's
// stream with no host synchronization when `fixed` (every radix level is
// launched and exits on the device when it has nothing to do): the form a
// CUDA graph captures.  *d_ng_out receives the device word of the group count.
int plan_pipeline(fmcs_ctx *ctx, const Plan &plan, const void *const *dcols, const uint32_t *col_bytes,
                  const uint32_t *bw, uint64_t n, bool hash, uint32_t *dorder, uint32_t *dgroup_out, bool fixed,
                  uint32_t **d_ng_out, const uint8_t *descending = nullptr)
{
    int rc;
    void *p;
    const uint32_t nbanks = (uint32_t)plan.banks.size();
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    // group ping-pong and segment starts
    uint32_t *g[2];
    if ((rc = ws_get(ctx, kSlotGroupA, n * 4, &p))) return rc;
    g[0] = (uint32_t *)p;
    if ((rc = ws_get(ctx, kSlotGroupB, n * 4, &p))) return rc;
    g[1] = (uint32_t *)p;
    uint32_t *segs[2];
    if ((rc = ws_get(ctx, kSlotSegStart, 2 * carve_round((n + 2) * sizeof(uint32_t)), &p))) return rc;
    {
        Carver cv(p);
        segs[0] = cv.take<uint32_t>(n + 2);
        segs[1] = cv.take<uint32_t>(n + 2);
    }
    uint32_t *d_nseg[2] = {w + kCtrNgroups + 2, w + kCtrNgroups + 3};
    const uint32_t *in_group = nullptr;
    const uint32_t *seg_in = nullptr;
    const uint32_t *d_nseg_in = nullptr;
    // (a) a bank's stitch reads only the columns: the next round's bank is
    // stitched on the context's second stream while this round sorts (its
    // buffer held the bank of the round before, finished by then)
    const uint32_t chunk_rows = msd_chunk_rows(ctx);
    uint32_t *top_hist = nullptr;
    auto stitch_bank = [&](uint32_t b, cudaStream_t s, void **bank_out) -> int {
        const BankPlan &bp = plan.banks[b];
        int r;
        if ((r = ws_get(ctx, kSlotBank0 + (b & 1), n * bp.bytes, bank_out))) return r;
        std::vector<StitchSlice> sl(bp.slices.size());
        for (size_t k = 0; k < bp.slices.size(); ++k) {
            const SliceRec &sr = bp.slices[k];
            sl[k] = StitchSlice{dcols[sr.col], col_bytes[sr.col], bw[sr.col] - sr.end, sr.end - sr.start + 1,
                                descending && descending[sr.col] ? 1u : 0u};
        }
        // round 0 of a sort plan over more rows than one block sorts: the
        // stitch also counts the first radix level's histograms
        uint32_t *th = nullptr;
        if (!hash && b == 0 && n > ctx->local_max) {
            const uint64_t nchunks = (n + chunk_rows - 1) / chunk_rows;
            void *q;
            if ((r = ws_get(ctx, kSlotTopHist, (nchunks + 1) * 256 * sizeof(uint32_t), &q))) return r;
            th = (uint32_t *)q;
            top_hist = th;
        }
        return launch_stitch(ctx, sl.data(), (int)sl.size(), *bank_out, bp.bytes, n, th, bp.bits, chunk_rows, s);
    };
    void *next_bank = nullptr;   // the next round's bank, stitched on the second stream
    for (uint32_t b = 0; b < nbanks; ++b) {
        const BankPlan &bp = plan.banks[b];
        const bool last = (b + 1 == nbanks);
        ctx->prof_round = (int)b;
        void *bank;
        if (next_bank) {
            bank = next_bank;
            next_bank = nullptr;
            if ((rc = join_par(ctx, ctx->stream))) return rc;
        } else if ((rc = stitch_bank(b, nullptr, &bank))) {
            return rc;
        }
        if (!last && !ctx->prof_on) {
            if ((rc = fork_par(ctx, ctx->stream))) return rc;
            if ((rc = stitch_bank(b + 1, ctx->par, &next_bank))) return rc;
        }
        if (b > 0) top_hist = nullptr;
        uint32_t *og = last ? (uint32_t *)(dgroup_out ? dgroup_out : g[b & 1]) : g[b & 1];
        if (!hash) {
            // (b)+(d): sort, then group ids (+ the next round's segments)
            uint32_t *ns = last ? nullptr : segs[b & 1];
            if ((rc = sort_round_dev(ctx, bank, bp.bytes, bp.bits, dorder, in_group, seg_in, d_nseg_in, og, nullptr,
                                     ns, d_nseg[b & 1], n, d_ng, false, fixed, top_hist)))
                return rc;
            seg_in = ns;
            d_nseg_in = d_nseg[b & 1];
        } else {
            // (e): hash grouping rounds; the last round leaves the order alone
            uint32_t *oin = in_group ? dorder : nullptr;
            if (!in_group && last) {
                if ((rc = launch_iota(ctx, dorder, n))) return rc;
                oin = dorder;
            }
            if ((rc = hash_round(ctx, bank, bp.bytes, oin, dorder, in_group, og, n, last, d_ng, false, fixed)))
                return rc;
        }
        in_group = og;
    }
    ctx->prof_round = -1;
    *d_ng_out = d_ng;
    return FMCS_OK;
}

}  // namespace
}  // namespace fmcs

using namespace fmcs;

extern "C" int fmcs_stitch(fmcs_ctx *ctx, const fmcs_slice *slices, uint32_t nslices, void *bank,
                           uint32_t bank_bytes, uint64_t n)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!slices || nslices == 0 || nslices > (uint32_t)kMaxSlices || !valid_bank(bank_bytes) || (!bank && n))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_stitch: invalid arguments");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_stitch: n must be < 2^32");
    std::vector<StitchSlice> sl(nslices);
    size_t stage_bytes = 0;
    for (uint32_t i = 0; i < nslices; ++i) {
        const fmcs_slice &s = slices[i];
        if (!valid_bank(s.src_bytes) || s.src_bits == 0 || s.src_bits > 8 * s.src_bytes || s.start < 1 ||
            s.end < s.start || s.end > s.src_bits || (!s.src && n))
            return set_error(ctx, FMCS_E_INVAL, "fmcs_stitch: invalid slice");
        if (!is_device_ptr(s.src)) stage_bytes += ((n * s.src_bytes + 255) & ~uint64_t(255));
    }
    int rc;
    char *stage = nullptr;
    if (stage_bytes) {
        void *p;
        if ((rc = ws_get(ctx, kSlotColStage, stage_bytes, &p))) return rc;
        stage = (char *)p;
    }
    for (uint32_t i = 0; i < nslices; ++i) {
        const fmcs_slice &s = slices[i];
        const void *src = s.src;
        if (!is_device_ptr(src)) {
            cudaError_t e = cudaMemcpyAsync(stage, src, n * s.src_bytes, cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_stitch stage");
            src = stage;
            stage += ((n * s.src_bytes + 255) & ~uint64_t(255));
        }
        sl[i] = StitchSlice{src, s.src_bytes, s.src_bits - s.end, s.end - s.start + 1, 0u};
    }
    void *dbank;
    bool host_out;
    if ((rc = stage_out(ctx, bank, n * bank_bytes, kSlotStageOut0, &dbank, &host_out))) return rc;
    if ((rc = launch_stitch(ctx, sl.data(), (int)nslices, dbank, bank_bytes, n))) return rc;
    if (host_out && (rc = copy_out(ctx, bank, dbank, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_stitch", nullptr, nullptr);
}

extern "C" int fmcs_shift_left(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n, uint32_t nbits)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!valid_bank(bank_bytes) || (n && !bank)) return set_error(ctx, FMCS_E_INVAL, "fmcs_shift_left: invalid arguments");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_shift_left: n must be < 2^32");
    if (n == 0) return FMCS_OK;
    int rc;
    void *dbank;
    bool host;
    if ((rc = stage_out(ctx, bank, n * bank_bytes, kSlotStageOut0, &dbank, &host))) return rc;
    if (host) {
        cudaError_t e = cudaMemcpyAsync(dbank, bank, n * bank_bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_shift_left stage");
    }
    if ((rc = launch_bank_update(ctx, dbank, bank_bytes, n, nbits, nullptr, 0, 0, 0))) return rc;
    if (host && (rc = copy_out(ctx, bank, dbank, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_shift_left", nullptr, nullptr);
}

extern "C" int fmcs_assemble(fmcs_ctx *ctx, void *bank, uint32_t bank_bytes, uint64_t n, const fmcs_slice *s)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!valid_bank(bank_bytes) || !s || (n && (!bank || !s->src)) || !valid_bank(s->src_bytes) || s->src_bits == 0 ||
        s->src_bits > 8 * s->src_bytes || s->start < 1 || s->end < s->start || s->end > s->src_bits)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_assemble: invalid arguments");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_assemble: n must be < 2^32");
    if (n == 0) return FMCS_OK;
    int rc;
    const void *dsrc = nullptr;
    if ((rc = stage_in(ctx, s->src, n * s->src_bytes, kSlotStageIn0, &dsrc))) return rc;
    void *dbank;
    bool host;
    if ((rc = stage_out(ctx, bank, n * bank_bytes, kSlotStageOut0, &dbank, &host))) return rc;
    if (host) {
        cudaError_t e = cudaMemcpyAsync(dbank, bank, n * bank_bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_assemble stage");
    }
    if ((rc = launch_bank_update(ctx, dbank, bank_bytes, n, 0, dsrc, s->src_bytes, s->src_bits - s->end,
                                 s->end - s->start + 1)))
        return rc;
    if (host && (rc = copy_out(ctx, bank, dbank, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_assemble", nullptr, nullptr);
}

extern "C" int fmcs_gather(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, const uint32_t *order, void *out,
                           uint64_t n)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!valid_bank(bank_bytes) || (n && (!bank || !order || !out)))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_gather: invalid arguments");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_gather: n must be < 2^32");
    if (n == 0) return FMCS_OK;
    int rc;
    const void *dbank = nullptr, *dorder = nullptr;
    if ((rc = stage_in(ctx, bank, n * bank_bytes, kSlotStageIn0, &dbank))) return rc;
    if ((rc = stage_in(ctx, order, n * 4, kSlotStageIn1, &dorder))) return rc;
    void *dout;
    bool host_out;
    if ((rc = stage_out(ctx, out, n * bank_bytes, kSlotStageOut0, &dout, &host_out))) return rc;
    if ((rc = launch_gather(ctx, dbank, bank_bytes, (const uint32_t *)dorder, dout, n))) return rc;
    if (host_out && (rc = copy_out(ctx, out, dout, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_gather", nullptr, nullptr);
}

extern "C" int fmcs_sort_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t key_bits,
                               uint32_t *order, const uint32_t *in_group, uint32_t *out_group, void *sorted_bank,
                               uint64_t n, uint32_t *ngroups)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (ngroups) *ngroups = 0;
    if (!(bank_bytes == 2 || bank_bytes == 4 || bank_bytes == 8))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round: bank_bytes must be 2, 4 or 8");
    if (key_bits == 0 || key_bits > 8 * bank_bytes)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round: key_bits must be in 1..8*bank_bytes");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round: n must be < 2^32");
    if (n == 0) return FMCS_OK;
    if (!bank || !order) return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round: bank and order are required");
    int rc;
    const void *dbank = nullptr, *dig = nullptr;
    if ((rc = stage_in(ctx, bank, n * bank_bytes, kSlotStageIn0, &dbank))) return rc;
    if ((rc = stage_in(ctx, in_group, n * 4, kSlotStageIn1, &dig))) return rc;
    void *dorder, *dgroup, *dkeys;
    bool h_order, h_group, h_keys;
    if ((rc = stage_out(ctx, order, n * 4, kSlotStageOut0, &dorder, &h_order))) return rc;
    if (h_order && in_group) {
        cudaError_t e = cudaMemcpyAsync(dorder, order, n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_sort_round stage order");
    }
    if ((rc = stage_out(ctx, out_group, n * 4, kSlotStageOut1, &dgroup, &h_group))) return rc;
    if ((rc = stage_out(ctx, sorted_bank, n * bank_bytes, kSlotStageOut2, &dkeys, &h_keys))) return rc;
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    if ((rc = sort_round_dev(ctx, dbank, bank_bytes, key_bits, (uint32_t *)dorder, (const uint32_t *)dig, nullptr,
                             nullptr, (uint32_t *)dgroup, dkeys, nullptr, nullptr, n, d_ng)))
        return rc;
    if (h_order && (rc = copy_out(ctx, order, dorder, n * 4))) return rc;
    if (h_group && (rc = copy_out(ctx, out_group, dgroup, n * 4))) return rc;
    if (h_keys && (rc = copy_out(ctx, sorted_bank, dkeys, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_sort_round", ngroups, out_group ? d_ng : nullptr);
}

extern "C" int fmcs_sort_round_plain(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t key_bits,
                                     uint32_t *order, const uint32_t *in_group, uint32_t *out_group,
                                     void *sorted_bank, uint64_t n, uint32_t *ngroups)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (ngroups) *ngroups = 0;
    if (!(bank_bytes == 2 || bank_bytes == 4 || bank_bytes == 8) || key_bits == 0 || key_bits > 8 * bank_bytes)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round_plain: bad bank width or key_bits");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round_plain: n must be < 2^32");
    if (n == 0) return FMCS_OK;
    if (!bank || !order) return set_error(ctx, FMCS_E_INVAL, "fmcs_sort_round_plain: bank and order are required");
    int rc;
    void *p;
    const void *dbank = nullptr, *dig = nullptr;
    if ((rc = stage_in(ctx, bank, n * bank_bytes, kSlotStageIn0, &dbank))) return rc;
    if ((rc = stage_in(ctx, in_group, n * 4, kSlotStageIn1, &dig))) return rc;
    void *dorder, *dgroup, *dkeys;
    bool h_order, h_group, h_keys;
    if ((rc = stage_out(ctx, order, n * 4, kSlotStageOut0, &dorder, &h_order))) return rc;
    if (h_order && in_group) {
        cudaError_t e = cudaMemcpyAsync(dorder, order, n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_sort_round_plain stage order");
    }
    if ((rc = stage_out(ctx, out_group, n * 4, kSlotStageOut1, &dgroup, &h_group))) return rc;
    if ((rc = stage_out(ctx, sorted_bank, n * bank_bytes, kSlotStageOut2, &dkeys, &h_keys))) return rc;
    void *kg;
    if ((rc = ws_get(ctx, kSlotKeys0, n * bank_bytes, &kg))) return rc;
    if ((rc = ws_get(ctx, kSlotMisc, 3 * carve_round(n * sizeof(uint32_t)), &p))) return rc;
    Carver cv(p);
    uint32_t *pos = cv.take<uint32_t>(n), *grp = cv.take<uint32_t>(n), *tmp = cv.take<uint32_t>(n);
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    cudaStream_t st = ctx->stream;
    // keys of this round in the previous order, positions as payload
    if (in_group) {
        if ((rc = launch_gather(ctx, dbank, bank_bytes, (const uint32_t *)dorder, kg, n))) return rc;
    } else {
        cudaMemcpyAsync(kg, dbank, n * bank_bytes, cudaMemcpyDeviceToDevice, st);
    }
    if ((rc = launch_iota(ctx, pos, n))) return rc;
    // full-array passes over the key, then (later rounds) over the group id
    if ((rc = lsd_sort_full(ctx, kg, bank_bytes, pos, n, key_bits))) return rc;
    if (in_group) {
        if ((rc = launch_gather(ctx, dig, 4, pos, grp, n))) return rc;
        cudaMemcpyAsync(ctx->h_small + 2, (const uint32_t *)dig + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_sort_round_plain sync");
        uint32_t gbits = 1;
        while (gbits < 32 && (1ull << gbits) <= (uint64_t)ctx->h_small[2]) gbits++;
        if ((rc = lsd_sort_full(ctx, grp, 4, pos, n, gbits))) return rc;
        // order_out[i] = order_in[pos[i]]
        cudaMemcpyAsync(tmp, dorder, n * 4, cudaMemcpyDeviceToDevice, st);
        if ((rc = launch_gather(ctx, tmp, 4, pos, dorder, n))) return rc;
        if ((rc = launch_gather(ctx, dbank, bank_bytes, (const uint32_t *)dorder, kg, n))) return rc;
    } else {
        cudaMemcpyAsync(dorder, pos, n * 4, cudaMemcpyDeviceToDevice, st);
    }
    if (dkeys) cudaMemcpyAsync(dkeys, kg, n * bank_bytes, cudaMemcpyDeviceToDevice, st);
    if (dgroup && (rc = launch_group_ids(ctx, kg, bank_bytes, in_group ? grp : nullptr, (uint32_t *)dgroup, n, d_ng)))
        return rc;
    if (h_order && (rc = copy_out(ctx, order, dorder, n * 4))) return rc;
    if (h_group && (rc = copy_out(ctx, out_group, dgroup, n * 4))) return rc;
    if (h_keys && (rc = copy_out(ctx, sorted_bank, dkeys, n * bank_bytes))) return rc;
    return finish(ctx, "fmcs_sort_round_plain", ngroups, out_group ? d_ng : nullptr);
}

extern "C" int fmcs_hash_round(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes, uint32_t *order,
                               const uint32_t *in_group, uint32_t *out_group, uint64_t n, int last_round,
                               uint32_t *ngroups)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (ngroups) *ngroups = 0;
    if (!valid_bank(bank_bytes))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_hash_round: bank_bytes must be 1, 2, 4 or 8");
    if (n >= kHashMaxRows) return set_error(ctx, FMCS_E_INVAL, "fmcs_hash_round: n must be < 2^31");
    if (n == 0) return FMCS_OK;
    if (!bank || !order || (!last_round && !out_group))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_hash_round: bank, order and (unless last) out_group required");
    int rc;
    const void *dbank = nullptr, *dig = nullptr;
    if ((rc = stage_in(ctx, bank, n * bank_bytes, kSlotStageIn0, &dbank))) return rc;
    if ((rc = stage_in(ctx, in_group, n * 4, kSlotStageIn1, &dig))) return rc;
    void *dorder, *dgroup;
    bool h_order, h_group;
    if ((rc = stage_out(ctx, order, n * 4, kSlotStageOut0, &dorder, &h_order))) return rc;
    if (h_order && in_group) {
        cudaError_t e = cudaMemcpyAsync(dorder, order, n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_hash_round stage order");
    }
    if ((rc = stage_out(ctx, out_group, n * 4, kSlotStageOut1, &dgroup, &h_group))) return rc;
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    uint32_t *oin = in_group ? (uint32_t *)dorder : nullptr;
    if (!in_group && last_round) {
        // round 0 and last: the order stays iota
        if ((rc = launch_iota(ctx, (uint32_t *)dorder, n))) return rc;
        oin = (uint32_t *)dorder;
    }
    if ((rc = hash_round(ctx, dbank, bank_bytes, oin, (uint32_t *)dorder, (const uint32_t *)dig,
                         (uint32_t *)dgroup, n, last_round != 0, d_ng)))
        return rc;
    if (h_order && (rc = copy_out(ctx, order, dorder, n * 4))) return rc;
    if (h_group && (rc = copy_out(ctx, out_group, dgroup, n * 4))) return rc;
    return finish(ctx, "fmcs_hash_round", ngroups, d_ng);
}

extern "C" int fmcs_hash_round_unordered(fmcs_ctx *ctx, const void *bank, uint32_t bank_bytes,
                                         const uint32_t *in_group, uint32_t *out_group, uint64_t n,
                                         uint32_t *ngroups)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (ngroups) *ngroups = 0;
    if (!valid_bank(bank_bytes) || (n && (!bank || !out_group)))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_hash_round_unordered: invalid arguments");
    if (n >= kHashMaxRows)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_hash_round_unordered: n must be < 2^31");
    if (n == 0) return FMCS_OK;
    int rc;
    const void *dbank = nullptr, *dig = nullptr;
    if ((rc = stage_in(ctx, bank, n * bank_bytes, kSlotStageIn0, &dbank))) return rc;
    if ((rc = stage_in(ctx, in_group, n * 4, kSlotStageIn1, &dig))) return rc;
    void *dgroup;
    bool h_group;
    if ((rc = stage_out(ctx, out_group, n * 4, kSlotStageOut1, &dgroup, &h_group))) return rc;
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    if ((rc = hash_round(ctx, dbank, bank_bytes, nullptr, nullptr, (const uint32_t *)dig, (uint32_t *)dgroup, n, true,
                         d_ng, true)))
        return rc;
    if (h_group && (rc = copy_out(ctx, out_group, dgroup, n * 4))) return rc;
    return finish(ctx, "fmcs_hash_round_unordered", ngroups, d_ng);
}

namespace {
int run_plan_impl(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                  uint32_t ncols, const uint32_t *col_order, const uint8_t *descending, const uint32_t *split,
                  uint32_t nbanks, uint64_t n, int hash, uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (ngroups) *ngroups = 0;
    if (!cols || !col_bytes || !bw || !split || ncols == 0 || nbanks == 0 || ncols > kMaxPlanCols ||
        nbanks > kMaxPlanBanks)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: invalid arguments");
    if (n >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: n must be < 2^32");
    if (hash && n >= kHashMaxRows) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: hash plans take n < 2^31");
    if (n && !order_out) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: order_out is required");
    for (uint32_t c = 0; c < ncols; ++c) {
        if (!valid_bank(col_bytes[c]) || bw[c] == 0 || bw[c] > 8 * col_bytes[c] || (n && !cols[c]))
            return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: invalid column");
        if (!hash && col_bytes[c] == 1)   // src/stitch_composer.cpp:681-687
            return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: 8-bit columns are not sortable (hash only)");
    }
    std::vector<uint32_t> corder(ncols);
    for (uint32_t c = 0; c < ncols; ++c) corder[c] = col_order ? col_order[c] : c;
    Plan plan;
    std::string perr;
    if (!build_plan(bw, ncols, corder.data(), split, nbanks, hash != 0, plan, perr))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_run_plan: " + perr);
    if (n == 0) return FMCS_OK;
    int rc;
    void *p;
    // stage host columns once
    std::vector<const void *> dcols(ncols);
    size_t stage_bytes = 0;
    for (uint32_t c = 0; c < ncols; ++c)
        if (!is_device_ptr(cols[c])) stage_bytes += ((n * col_bytes[c] + 255) & ~uint64_t(255));
    char *stage = nullptr;
    if (stage_bytes) {
        if ((rc = ws_get(ctx, kSlotColStage, stage_bytes, &p))) return rc;
        stage = (char *)p;
    }
    for (uint32_t c = 0; c < ncols; ++c) {
        if (is_device_ptr(cols[c])) {
            dcols[c] = cols[c];
        } else {
            cudaError_t e = cudaMemcpyAsync(stage, cols[c], n * col_bytes[c], cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_plan stage");
            dcols[c] = stage;
            stage += ((n * col_bytes[c] + 255) & ~uint64_t(255));
        }
    }
    void *dorder, *dgroup_out;
    bool h_order, h_group;
    if ((rc = stage_out(ctx, order_out, n * 4, kSlotStageOut0, &dorder, &h_order))) return rc;
    if ((rc = stage_out(ctx, group_out, n * 4, kSlotStageOut1, &dgroup_out, &h_group))) return rc;
    uint32_t *d_ng = nullptr;
    if ((rc = plan_pipeline(ctx, plan, dcols.data(), col_bytes, bw, n, hash != 0, (uint32_t *)dorder,
                            (uint32_t *)dgroup_out, false, &d_ng, descending)))
        return rc;
    ctx->prof_round = -1;
    if (h_order && (rc = copy_out(ctx, order_out, dorder, n * 4))) return rc;
    if (h_group && (rc = copy_out(ctx, group_out, dgroup_out, n * 4))) return rc;
    return finish(ctx, "fmcs_run_plan", ngroups, d_ng);
}
}  // namespace

extern "C" int fmcs_run_plan(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                             uint32_t ncols, const uint32_t *col_order, const uint32_t *split, uint32_t nbanks,
                             uint64_t n, int hash, uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups)
{
    return run_plan_impl(ctx, cols, col_bytes, bw, ncols, col_order, nullptr, split, nbanks, n, hash, order_out,
                         group_out, ngroups);
}

extern "C" int fmcs_run_plan_desc(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes,
                                  const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                                  const uint8_t *descending, const uint32_t *split, uint32_t nbanks, uint64_t n,
                                  int hash, uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups)
{
    return run_plan_impl(ctx, cols, col_bytes, bw, ncols, col_order, descending, split, nbanks, n, hash, order_out,
                         group_out, ngroups);
}

// ---------------------------------------------------------------------------
// Many independent instances in one batch
// ---------------------------------------------------------------------------
namespace fmcs {
namespace {

__global__ void instance_ids_kernel(const uint32_t *starts, uint32_t ninst, uint32_t *inst_id, uint64_t n)
{
    kernel_prologue();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = ninst;   // starts[lo] <= i < starts[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (starts[mid] <= i) lo = mid; else hi = mid;
        }
        inst_id[i] = lo;
    }
}

__global__ void instance_bases_kernel(const uint32_t *starts, uint32_t ninst, const uint32_t *group, uint32_t *base,
                                      uint32_t *count)
{
    kernel_prologue();
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ninst; k += gridDim.x * blockDim.x) {
        const uint32_t s = starts[k], e = starts[k + 1];
        base[k] = e > s ? group[s] : 0u;
        count[k] = e > s ? group[e - 1] - group[s] + 1 : 0u;
    }
}

__global__ void localize_kernel(const uint32_t *starts, const uint32_t *inst_id, const uint32_t *base,
                                uint32_t *order, uint32_t *group, uint64_t n)
{
    kernel_prologue();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = inst_id[i];
        order[i] -= starts[k];
        if (group) group[i] -= base[k];
    }
}

}  // namespace
}  // namespace fmcs

extern "C" int fmcs_run_batch(fmcs_ctx *ctx, const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                              uint32_t ncols, const uint32_t *split, uint32_t nbanks, const fmcs_instance *inst,
                              uint32_t ninst, uint64_t total_rows, uint32_t *order_out, uint32_t *group_out,
                              uint32_t *ngroups_out)
{
    if (!ctx) return FMCS_E_INVAL;
    cudaSetDevice(ctx->device);
    if (!cols || !col_bytes || !bw || !split || !inst || ncols == 0 || nbanks == 0 || ninst == 0 ||
        ncols > kMaxPlanCols || nbanks > kMaxPlanBanks)
        return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: invalid arguments");
    if (total_rows >= (1ull << 32)) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: total_rows must be < 2^32");
    std::vector<uint32_t> starts(ninst + 1);
    uint64_t off = 0;
    for (uint32_t k = 0; k < ninst; ++k) {
        if (inst[k].row_off != off)
            return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: instances must be contiguous and in row order");
        starts[k] = (uint32_t)off;
        off += inst[k].n;
    }
    if (off != total_rows) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: instance rows do not add up");
    starts[ninst] = (uint32_t)off;
    for (uint32_t c = 0; c < ncols; ++c) {
        if (!valid_bank(col_bytes[c]) || col_bytes[c] == 1 || bw[c] == 0 || bw[c] > 8 * col_bytes[c] ||
            (total_rows && !cols[c]))
            return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: invalid column");
    }
    std::vector<uint32_t> corder(ncols);
    for (uint32_t c = 0; c < ncols; ++c) corder[c] = c;
    Plan plan;
    std::string perr;
    if (!build_plan(bw, ncols, corder.data(), split, nbanks, false, plan, perr))
        return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: " + perr);
    const uint64_t n = total_rows;
    if (n == 0) {
        if (ngroups_out)
            for (uint32_t k = 0; k < ninst; ++k) ngroups_out[k] = 0;
        return FMCS_OK;
    }
    if (!order_out) return set_error(ctx, FMCS_E_INVAL, "fmcs_run_batch: order_out is required");
    int rc;
    void *p;
    cudaStream_t st = ctx->stream;
    // instance starts, ids per row, bases and counts
    if ((rc = ws_get(ctx, kSlotMisc,
                     carve_total({(ninst + 1) * sizeof(uint32_t), ninst * sizeof(uint32_t),
                                  (ninst + 1) * sizeof(uint32_t), n * sizeof(uint32_t)}),
                     &p)))
        return rc;
    Carver cv(p);
    uint32_t *d_starts = cv.take<uint32_t>(ninst + 1);
    uint32_t *d_base = cv.take<uint32_t>(ninst);
    uint32_t *d_count = cv.take<uint32_t>(ninst + 1);
    uint32_t *inst_id = cv.take<uint32_t>(n);
    cudaError_t e = cudaMemcpyAsync(d_starts, starts.data(), (ninst + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_batch upload");
    {
        LaunchScope ls_(ctx, "instance_ids");
        launch_k(instance_ids_kernel, ctx->num_sms * 8, 256, 0, st, d_starts, ninst, inst_id, n);
    }
    uint32_t *w;
    if ((rc = counters(ctx, &w))) return rc;
    uint32_t *d_ng = w + kCtrNgroups;
    uint32_t *d_ninst = w + kCtrNgroups + 4;
    e = cudaMemcpyAsync(d_ninst, &ninst, sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_batch upload");
    // columns
    std::vector<const void *> dcols(ncols);
    size_t stage_bytes = 0;
    for (uint32_t c = 0; c < ncols; ++c)
        if (!is_device_ptr(cols[c])) stage_bytes += ((n * col_bytes[c] + 255) & ~uint64_t(255));
    char *stage = nullptr;
    if (stage_bytes) {
        if ((rc = ws_get(ctx, kSlotColStage, stage_bytes, &p))) return rc;
        stage = (char *)p;
    }
    for (uint32_t c = 0; c < ncols; ++c) {
        if (is_device_ptr(cols[c])) {
            dcols[c] = cols[c];
        } else {
            e = cudaMemcpyAsync(stage, cols[c], n * col_bytes[c], cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_batch stage");
            dcols[c] = stage;
            stage += ((n * col_bytes[c] + 255) & ~uint64_t(255));
        }
    }
    void *dorder, *dgroup_out;
    bool h_order, h_group;
    if ((rc = stage_out(ctx, order_out, n * 4, kSlotStageOut0, &dorder, &h_order))) return rc;
    if ((rc = stage_out(ctx, group_out, n * 4, kSlotStageOut1, &dgroup_out, &h_group))) return rc;
    uint32_t *g[2];
    if ((rc = ws_get(ctx, kSlotGroupA, n * 4, &p))) return rc;
    g[0] = (uint32_t *)p;
    if ((rc = ws_get(ctx, kSlotGroupB, n * 4, &p))) return rc;
    g[1] = (uint32_t *)p;
    uint32_t *segs[2];
    if ((rc = ws_get(ctx, kSlotSegStart, 2 * carve_round((n + 2) * sizeof(uint32_t)), &p))) return rc;
    {
        Carver cv(p);
        segs[0] = cv.take<uint32_t>(n + 2);
        segs[1] = cv.take<uint32_t>(n + 2);
    }
    uint32_t *d_nseg[2] = {w + kCtrNgroups + 2, w + kCtrNgroups + 3};
    // round 0 is segmented by instance: instance ids are the incoming groups
    const uint32_t *in_group = inst_id;
    const uint32_t *seg_in = d_starts;
    const uint32_t *d_nseg_in = d_ninst;
    for (uint32_t b = 0; b < nbanks; ++b) {
        const BankPlan &bp = plan.banks[b];
        const bool last = (b + 1 == nbanks);
        ctx->prof_round = (int)b;
        void *bank;
        if ((rc = ws_get(ctx, kSlotBank0 + (b & 1), n * bp.bytes, &bank))) return rc;
        std::vector<StitchSlice> sl(bp.slices.size());
        for (size_t k = 0; k < bp.slices.size(); ++k) {
            const SliceRec &r = bp.slices[k];
            sl[k] = StitchSlice{dcols[r.col], col_bytes[r.col], bw[r.col] - r.end, r.end - r.start + 1, 0u};
        }
        if ((rc = launch_stitch(ctx, sl.data(), (int)sl.size(), bank, bp.bytes, n))) return rc;
        uint32_t *og = (last && dgroup_out) ? (uint32_t *)dgroup_out : g[b & 1];
        uint32_t *ns = last ? nullptr : segs[b & 1];
        if ((rc = sort_round_dev(ctx, bank, bp.bytes, bp.bits, (uint32_t *)dorder, in_group, seg_in, d_nseg_in, og,
                                 nullptr, ns, d_nseg[b & 1], n, d_ng, b == 0)))
            return rc;
        seg_in = ns;
        d_nseg_in = d_nseg[b & 1];
        in_group = og;
    }
    ctx->prof_round = -1;
    // instance-local oids and group ids
    {
        LaunchScope ls_(ctx, "instance_bases");
        launch_k(instance_bases_kernel, (ninst + 255) / 256, 256, 0, st, d_starts, ninst, in_group, d_base, d_count);
    }
    {
        LaunchScope ls_(ctx, "localize");
        launch_k(localize_kernel, ctx->num_sms * 8, 256, 0, st, d_starts, inst_id, d_base, (uint32_t *)dorder,
                                                           (uint32_t *)in_group, n);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_batch localize");
    if (ngroups_out) {
        e = cudaMemcpyAsync(ngroups_out, d_count, ninst * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fmcs_run_batch counts");
    }
    if (h_order && (rc = copy_out(ctx, order_out, dorder, n * 4))) return rc;
    if (h_group && (rc = copy_out(ctx, group_out, dgroup_out, n * 4))) return rc;
    return finish(ctx, "fmcs_run_batch", nullptr, nullptr);
}

// ---------------------------------------------------------------------------
// A whole sort plan captured once as a CUDA graph and replayed
// ---------------------------------------------------------------------------
struct fmcs_graph {
    fmcs_ctx *ctx = nullptr;   // private context: its workspace stays as captured
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t *d_ng = nullptr;
    unsigned long long kernels = 0;   // kernel nodes captured (a loop body once)
};

extern "C" void fmcs_graph_destroy(fmcs_graph *g)
{
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->ctx) fmcs_destroy(g->ctx);
    delete g;
}

static int graph_create(fmcs_ctx *parent, const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                        uint32_t ncols, const uint32_t *col_order, const uint32_t *split, uint32_t nbanks, uint64_t n,
                        bool hash, uint32_t *order_out, uint32_t *group_out, fmcs_graph **out)
{
    if (!parent || !out) return FMCS_E_INVAL;
    *out = nullptr;
    cudaSetDevice(parent->device);
    if (!cols || !col_bytes || !bw || !split || ncols == 0 || nbanks == 0 || ncols > kMaxPlanCols ||
        nbanks > kMaxPlanBanks || n == 0 || n >= (hash ? kHashMaxRows : (1ull << 32)) || !order_out)
        return set_error(parent, FMCS_E_INVAL, "fmcs_graph_create: invalid arguments");
    for (uint32_t c = 0; c < ncols; ++c) {
        if (!(col_bytes[c] == 2 || col_bytes[c] == 4 || col_bytes[c] == 8) || bw[c] == 0 || bw[c] > 8 * col_bytes[c])
            return set_error(parent, FMCS_E_INVAL, "fmcs_graph_create: invalid column");
        if (!is_device_ptr(cols[c]))
            return set_error(parent, FMCS_E_INVAL, "fmcs_graph_create: columns must be device memory");
    }
    if (!is_device_ptr(order_out) || (group_out && !is_device_ptr(group_out)))
        return set_error(parent, FMCS_E_INVAL, "fmcs_graph_create: outputs must be device memory");
    std::vector<uint32_t> corder(ncols);
    for (uint32_t c = 0; c < ncols; ++c) corder[c] = col_order ? col_order[c] : c;
    Plan plan;
    std::string perr;
    if (!build_plan(bw, ncols, corder.data(), split, nbanks, hash, plan, perr))
        return set_error(parent, FMCS_E_INVAL, "fmcs_graph_create: " + perr);
    fmcs_graph *g = new fmcs_graph();
    int rc = fmcs_create(&g->ctx, parent->device, 0);
    if (rc) {
        delete g;
        return set_error(parent, rc, "fmcs_graph_create: context");
    }
    fmcs_ctx *ctx = g->ctx;
    ctx->rank_mode = parent->rank_mode;
    ctx->local_max = parent->local_max;
    ctx->msd_items = parent->msd_items;
    // 1) one eager run of the fixed launch sequence sizes every workspace slot
    rc = plan_pipeline(ctx, plan, cols, col_bytes, bw, n, hash, order_out, group_out, true, &g->d_ng);
    if (!rc) rc = check_status(ctx, "fmcs_graph_create warm-up");
    // 2) capture: reset the look-back words (their epochs repeat on every
    //    replay), then the same launches
    if (!rc) {
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int slot : {kSlotLookback, kSlotScanTiles})
                if (ctx->ws.ptr[slot]) cudaMemsetAsync(ctx->ws.ptr[slot], 0, ctx->ws.cap[slot], ctx->stream);
            const unsigned long long l0 = ctx->launches;   // every launch site counts itself
            rc = plan_pipeline(ctx, plan, cols, col_bytes, bw, n, hash, order_out, group_out, true, &g->d_ng);
            g->kernels = ctx->launches - l0;
            cudaGraph_t graph = nullptr;
            e = cudaStreamEndCapture(ctx->stream, &graph);
            g->graph = graph;
            if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, graph, 0);
        }
        if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "fmcs_graph_create capture");
    }
    if (rc) {
        set_error(parent, rc, std::string("fmcs_graph_create: ") + ctx->err);
        fmcs_graph_destroy(g);
        return rc;
    }
    *out = g;
    return FMCS_OK;
}

extern "C" int fmcs_graph_create(fmcs_ctx *parent, const void *const *cols, const uint32_t *col_bytes,
                                 const uint32_t *bw, uint32_t ncols, const uint32_t *col_order, const uint32_t *split,
                                 uint32_t nbanks, uint64_t n, uint32_t *order_out, uint32_t *group_out,
                                 fmcs_graph **out)
{
    return graph_create(parent, cols, col_bytes, bw, ncols, col_order, split, nbanks, n, false, order_out, group_out,
                        out);
}

extern "C" int fmcs_graph_create_hash(fmcs_ctx *parent, const void *const *cols, const uint32_t *col_bytes,
                                      const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                                      const uint32_t *split, uint32_t nbanks, uint64_t n, uint32_t *order_out,
                                      uint32_t *group_out, fmcs_graph **out)
{
    return graph_create(parent, cols, col_bytes, bw, ncols, col_order, split, nbanks, n, true, order_out, group_out,
                        out);
}

extern "C" int fmcs_graph_launch(fmcs_graph *g, uint32_t *ngroups)
{
    if (!g || !g->exec) return FMCS_E_INVAL;
    cudaSetDevice(g->ctx->device);
    cudaError_t e = cudaGraphLaunch(g->exec, g->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(g->ctx, e, "fmcs_graph_launch");
    return finish(g->ctx, "fmcs_graph_launch", ngroups, g->d_ng);
}

extern "C" void *fmcs_graph_stream(fmcs_graph *g) { return g && g->ctx ? (void *)g->ctx->stream : nullptr; }

extern "C" int fmcs_graph_kernels(fmcs_graph *g)
{
    if (!g || !g->graph) return -1;
    return (int)g->kernels;
}
