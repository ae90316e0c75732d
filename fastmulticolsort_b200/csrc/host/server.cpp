// server.cpp -- the serving loop of include/fmcs_server.h: execution slots
// (worker threads with their own context and stream), admission against an
// HBM budget, and continuous batching of small compatible requests into one
// fmcs_run_batch launch.
#include "../../../include/fmcs_server.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Pending {
    uint64_t ticket = 0;
    fmcs_request req{};
    std::vector<const void *> cols;
    std::vector<uint32_t> col_bytes, bw, split;
    size_t footprint = 0;
    Clock::time_point submitted, started, finished;
    fmcs_result result{};
    bool done = false;
};

// Device bytes one request needs while it runs (banks, sort buffers, group
// vectors, segment lists; hash rounds add their table).
size_t footprint_of(const fmcs_request &r, const std::vector<uint32_t> &split)
{
    uint32_t maxb = 2;
    for (uint32_t w : split) maxb = std::max<uint32_t>(maxb, w <= 16 ? 2 : (w <= 32 ? 4 : 8));
    size_t per_row = 3 * maxb + 64 + (r.hash ? 32 : 0);
    for (uint32_t c = 0; c < r.ncols; ++c) {
        cudaPointerAttributes a;
        const bool dev = cudaPointerGetAttributes(&a, r.cols[c]) == cudaSuccess &&
                         (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
        if (!dev) {
            cudaGetLastError();
            per_row += r.col_bytes[c];   // staged copy
        }
    }
    return (size_t)r.n * per_row + (1u << 20);
}

bool compatible(const Pending &a, const Pending &b)
{
    return a.req.hash == 0 && b.req.hash == 0 && a.bw == b.bw && a.col_bytes == b.col_bytes && a.split == b.split;
}

}  // namespace

struct fmcs_server {
    int device = 0;
    size_t budget = 0;
    uint64_t batch_rows_max = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Pending>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Pending>> tickets;
    size_t admitted = 0;
    uint32_t running = 0;
    bool stop = false;
    uint64_t next_ticket = 1;
    std::vector<std::thread> workers;
};

namespace {

struct Staging {
    void *ptr = nullptr;
    size_t cap = 0;
    void *get(size_t bytes)
    {
        if (cap >= bytes) return ptr;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        if (cudaMalloc(&ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cap = bytes;
        return ptr;
    }
    ~Staging()
    {
        if (ptr) cudaFree(ptr);
    }
};

void run_alone(fmcs_ctx *ctx, Pending &p)
{
    uint32_t ng = 0;
    const int rc = fmcs_run_plan(ctx, p.cols.data(), p.col_bytes.data(), p.bw.data(), p.req.ncols, nullptr,
                                 p.split.data(), (uint32_t)p.split.size(), p.req.n, p.req.hash, p.req.order_out,
                                 p.req.group_out, &ng);
    p.result.status = rc;
    p.result.ngroups = ng;
    p.result.batched_with = 1;
}

void run_batched(fmcs_ctx *ctx, std::vector<std::shared_ptr<Pending>> &group, Staging &cols_stage, Staging &out_stage)
{
    const Pending &h = *group[0];
    const uint32_t ncols = h.req.ncols;
    uint64_t total = 0;
    for (auto &p : group) total += p->req.n;
    size_t col_bytes_total = 0;
    std::vector<size_t> col_off(ncols);
    for (uint32_t c = 0; c < ncols; ++c) {
        col_off[c] = col_bytes_total;
        col_bytes_total += ((total * h.col_bytes[c] + 255) & ~size_t(255));
    }
    char *cbase = (char *)cols_stage.get(col_bytes_total);
    uint32_t *obase = (uint32_t *)out_stage.get(2 * total * sizeof(uint32_t) + 256);
    int rc = (cbase && obase) ? FMCS_OK : FMCS_E_OOM;
    cudaStream_t st = (cudaStream_t)fmcs_stream(ctx);
    std::vector<fmcs_instance> inst(group.size());
    uint64_t off = 0;
    for (size_t k = 0; k < group.size() && rc == FMCS_OK; ++k) {
        const Pending &p = *group[k];
        inst[k] = fmcs_instance{off, p.req.n};
        for (uint32_t c = 0; c < ncols; ++c) {
            if (cudaMemcpyAsync(cbase + col_off[c] + off * h.col_bytes[c], p.cols[c], p.req.n * h.col_bytes[c],
                                cudaMemcpyDefault, st) != cudaSuccess)
                rc = FMCS_E_CUDA;
        }
        off += p.req.n;
    }
    std::vector<const void *> cols(ncols);
    for (uint32_t c = 0; c < ncols; ++c) cols[c] = cbase + col_off[c];
    std::vector<uint32_t> counts(group.size(), 0);
    uint32_t *order = obase, *grp = obase + total;
    if (rc == FMCS_OK)
        rc = fmcs_run_batch(ctx, cols.data(), h.col_bytes.data(), h.bw.data(), ncols, h.split.data(),
                            (uint32_t)h.split.size(), inst.data(), (uint32_t)group.size(), total, order, grp,
                            counts.data());
    for (size_t k = 0; k < group.size() && rc == FMCS_OK; ++k) {
        Pending &p = *group[k];
        if (cudaMemcpyAsync(p.req.order_out, order + inst[k].row_off, p.req.n * 4, cudaMemcpyDefault, st) !=
                cudaSuccess ||
            (p.req.group_out && cudaMemcpyAsync(p.req.group_out, grp + inst[k].row_off, p.req.n * 4,
                                                cudaMemcpyDefault, st) != cudaSuccess))
            rc = FMCS_E_CUDA;
    }
    if (rc == FMCS_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = FMCS_E_CUDA;
    for (size_t k = 0; k < group.size(); ++k) {
        group[k]->result.status = rc;
        group[k]->result.ngroups = counts[k];
        group[k]->result.batched_with = (uint32_t)group.size();
    }
}

void worker(fmcs_server *s)
{
    cudaSetDevice(s->device);
    fmcs_ctx *ctx = nullptr;
    const int crc = fmcs_create(&ctx, s->device, 0);
    Staging cols_stage, out_stage;
    for (;;) {
        std::vector<std::shared_ptr<Pending>> group;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                return s->stop ||
                       (!s->queue.empty() && (s->admitted == 0 || s->admitted + s->queue.front()->footprint <= s->budget));
            });
            if (s->queue.empty()) break;   // stop requested and nothing admitted-able left
            if (s->stop) break;
            auto head = s->queue.front();
            s->queue.pop_front();
            group.push_back(head);
            size_t fp = head->footprint;
            if (head->req.n <= s->batch_rows_max && head->req.hash == 0) {
                uint64_t rows = head->req.n;
                for (auto it = s->queue.begin(); it != s->queue.end();) {
                    Pending &q = **it;
                    if (q.req.n <= s->batch_rows_max && compatible(*head, q) && rows + q.req.n <= s->batch_rows_max &&
                        s->admitted + fp + q.footprint <= s->budget) {
                        rows += q.req.n;
                        fp += q.footprint;
                        group.push_back(*it);
                        it = s->queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            s->admitted += fp;
            s->running += (uint32_t)group.size();
            const auto now = Clock::now();
            for (auto &p : group) p->started = now;
        }
        if (crc != FMCS_OK) {
            for (auto &p : group) p->result.status = crc;
        } else if (group.size() == 1) {
            run_alone(ctx, *group[0]);
        } else {
            run_batched(ctx, group, cols_stage, out_stage);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            const auto now = Clock::now();
            for (auto &p : group) {
                s->admitted -= p->footprint;
                p->finished = now;
                p->result.queue_ms = ms_between(p->submitted, p->started);
                p->result.run_ms = ms_between(p->started, p->finished);
                p->result.total_ms = ms_between(p->submitted, p->finished);
                p->done = true;
            }
            s->running -= (uint32_t)group.size();
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    if (ctx) fmcs_destroy(ctx);
}

}  // namespace

extern "C" int fmcs_server_create(fmcs_server **out, int device, size_t hbm_budget_bytes, uint32_t slots,
                                  uint64_t batch_rows_max)
{
    if (!out || slots == 0 || slots > 64) return FMCS_E_INVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return FMCS_E_CUDA;
    }
    fmcs_server *s = new fmcs_server();
    s->device = device;
    s->budget = hbm_budget_bytes ? hbm_budget_bytes : ~size_t(0);
    s->batch_rows_max = batch_rows_max;
    for (uint32_t i = 0; i < slots; ++i) s->workers.emplace_back(worker, s);
    *out = s;
    return FMCS_OK;
}

extern "C" int fmcs_server_submit(fmcs_server *s, const fmcs_request *req, uint64_t *ticket)
{
    if (!s || !req || !ticket || !req->cols || !req->col_bytes || !req->bw || req->ncols == 0 || req->ncols > 64 ||
        (req->n && !req->order_out) || req->n >= (1ull << 32))
        return FMCS_E_INVAL;
    auto p = std::make_shared<Pending>();
    p->req = *req;
    p->cols.assign(req->cols, req->cols + req->ncols);
    p->col_bytes.assign(req->col_bytes, req->col_bytes + req->ncols);
    p->bw.assign(req->bw, req->bw + req->ncols);
    if (req->split && req->nbanks) {
        p->split.assign(req->split, req->split + req->nbanks);
    } else {
        std::vector<uint64_t> card(req->ncols);
        for (uint32_t c = 0; c < req->ncols; ++c)
            card[c] = req->cardinality ? req->cardinality[c]
                                       : std::min<uint64_t>(req->n ? req->n : 1, req->bw[c] >= 63 ? ~0ull : (1ull << req->bw[c]));
        uint32_t split[64], nb = 0;
        const int rc = fmcs_optimize_plan(req->bw, card.data(), req->col_bytes, req->ncols, req->n ? req->n : 1, 1,
                                          split, 64, &nb, nullptr, nullptr);
        if (rc != FMCS_OK) return rc;
        p->split.assign(split, split + nb);
    }
    p->footprint = footprint_of(*req, p->split);
    if (p->footprint > s->budget) return FMCS_E_OOM;
    p->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return FMCS_E_INVAL;
        p->ticket = s->next_ticket++;
        *ticket = p->ticket;
        s->tickets[p->ticket] = p;
        s->queue.push_back(p);
    }
    s->cv_work.notify_one();
    return FMCS_OK;
}

extern "C" int fmcs_server_wait(fmcs_server *s, uint64_t ticket, double timeout_s, fmcs_result *result)
{
    if (!s) return FMCS_E_INVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return FMCS_E_INVAL;
    auto p = it->second;
    auto ready = [&] { return p->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return FMCS_E_TIMEOUT;
    }
    if (result) *result = p->result;
    s->tickets.erase(ticket);
    return FMCS_OK;
}

extern "C" int fmcs_server_load(fmcs_server *s, size_t *admitted, uint32_t *queued, uint32_t *running)
{
    if (!s) return FMCS_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (admitted) *admitted = s->admitted;
    if (queued) *queued = (uint32_t)s->queue.size();
    if (running) *running = s->running;
    return FMCS_OK;
}

extern "C" void fmcs_server_destroy(fmcs_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto &p : s->queue) {
            p->result.status = FMCS_E_INVAL;
            p->done = true;
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto &t : s->workers) t.join();
    delete s;
}
