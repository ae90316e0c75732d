// composer.cpp -- Column helpers, the per-thread default context, and the
// Composer / ChainComposer round engines (include/fmcs/composer.h) on top of
// the C ABI.
//
// Reference: src/composer.cpp (multiRoundSorting :48-135, the hash round
// loops :137-381, sortByGroup :1222-1408) and src/chain_composer.cpp:12-25.
#include "../../../include/fmcs/composer.h"

#include <cuda_runtime.h>

#include <chrono>
#include <stdexcept>
#include <string>

namespace multiAttrSort {

// ---------------------------------------------------------------- context
namespace {

struct ThreadContext {
    fmcs_ctx *ctx = nullptr;
    int device = -1;
    ~ThreadContext()
    {
        if (ctx) fmcs_destroy(ctx);
    }
};

thread_local ThreadContext t_ctx;

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

fmcs_ctx *DefaultContext()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    if (!t_ctx.ctx || t_ctx.device != dev) {
        if (t_ctx.ctx) fmcs_destroy(t_ctx.ctx);
        t_ctx.ctx = nullptr;
        int rc = fmcs_create(&t_ctx.ctx, dev, 0);
        if (rc != FMCS_OK) throw std::runtime_error("fmcs: cannot create a context on device " + std::to_string(dev));
        t_ctx.device = dev;
    }
    return t_ctx.ctx;
}

namespace detail {

static bool on_device(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void elem_read(const void *base, uint64_t idx, uint32_t bytes, void *out)
{
    const char *p = (const char *)base + idx * bytes;
    if (on_device(base)) {
        if (cudaMemcpy(out, p, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("fmcs: element read failed");
    } else {
        for (uint32_t i = 0; i < bytes; ++i) ((char *)out)[i] = p[i];
    }
}

void elem_write(void *base, uint64_t idx, uint32_t bytes, const void *in)
{
    char *p = (char *)base + idx * bytes;
    if (on_device(base)) {
        if (cudaMemcpy(p, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("fmcs: element write failed");
    } else {
        for (uint32_t i = 0; i < bytes; ++i) p[i] = ((const char *)in)[i];
    }
}

void check(int rc, const char *what)
{
    if (rc != FMCS_OK) {
        const char *msg = t_ctx.ctx ? fmcs_last_error(t_ctx.ctx) : "";
        throw std::runtime_error(std::string("fmcs: ") + what + " failed (" + std::to_string(rc) + "): " + msg);
    }
}

}  // namespace detail

// ---------------------------------------------------------------- Composer
Composer::Composer(setting_t setting, uint32_t ncolumns, uint64_t nrows, compose_params_t params,
                   Column **column_values)
    : num_columns_(ncolumns), num_rows_(nrows), column_values_(column_values), setting_(setting),
      compose_params_(params)
{
}

Composer::Composer() : num_columns_(0), num_rows_(0), column_values_(nullptr) {}

Composer::~Composer()
{
    if (d_order_) cudaFree(d_order_);
    if (d_group_[0]) cudaFree(d_group_[0]);
    if (d_group_[1]) cudaFree(d_group_[1]);
}

fmcs_ctx *Composer::GetContext() { return ctx_ ? ctx_ : DefaultContext(); }

void Composer::SortAllColumns()
{
    switch (compose_params_.packtype) {
    case PackOIDType::pack: SortAllColumns_Pack(); break;
    case PackOIDType::nonpack: SortAllColumns_Nonpack(); break;
    }
}

void Composer::ensure_buffers()
{
    if (buf_rows_ >= num_rows_ && d_order_) return;
    if (d_order_) cudaFree(d_order_);
    if (d_group_[0]) cudaFree(d_group_[0]);
    if (d_group_[1]) cudaFree(d_group_[1]);
    d_order_ = d_group_[0] = d_group_[1] = nullptr;
    const size_t bytes = (num_rows_ ? num_rows_ : 1) * sizeof(surrogate_t);
    if (cudaMalloc(&d_order_, bytes) != cudaSuccess || cudaMalloc(&d_group_[0], bytes) != cudaSuccess ||
        cudaMalloc(&d_group_[1], bytes) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("fmcs: cannot allocate the composer's order / group buffers");
    }
    buf_rows_ = num_rows_;
}

std::vector<surrogate_t> Composer::GetOrder() const
{
    std::vector<surrogate_t> v(num_rows_);
    if (num_rows_) CopyOrderTo(v.data());
    return v;
}

std::vector<surrogate_t> Composer::GetGroup() const
{
    std::vector<surrogate_t> v(num_rows_);
    if (num_rows_) CopyGroupTo(v.data());
    return v;
}

void Composer::CopyOrderTo(surrogate_t *dst) const
{
    if (!d_order_) throw std::runtime_error("fmcs: no result yet");
    if (cudaMemcpy(dst, d_order_, num_rows_ * sizeof(surrogate_t), cudaMemcpyDefault) != cudaSuccess)
        throw std::runtime_error("fmcs: copy of the order failed");
}

void Composer::CopyGroupTo(surrogate_t *dst) const
{
    if (!d_group_[final_group_]) throw std::runtime_error("fmcs: no result yet");
    if (cudaMemcpy(dst, d_group_[final_group_], num_rows_ * sizeof(surrogate_t), cudaMemcpyDefault) != cudaSuccess)
        throw std::runtime_error("fmcs: copy of the group ids failed");
}

void Composer::sort_round_any(surrogate_t *outGroup, void *inValues, uint32_t bytes, surrogate_t *order,
                              surrogate_t *inGroup, uint32_t bitwidth, bool isLastRound)
{
    uint32_t ng = 0;
    // round 0 sorts the caller's values in place, as the reference does
    void *sorted = inGroup ? nullptr : inValues;
    detail::check(fmcs_sort_round(GetContext(), inValues, bytes, bitwidth, order, inGroup,
                                  isLastRound ? nullptr : outGroup, sorted, num_rows_, &ng),
                  "sortByGroup");
}

void *Composer::gather_any(const void *values, uint32_t bytes, const surrogate_t *order)
{
    void *out = nullptr;
    if (cudaMalloc(&out, (num_rows_ ? num_rows_ : 1) * bytes) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("fmcs: BATproject allocation failed");
    }
    detail::check(fmcs_gather(GetContext(), values, bytes, order, out, num_rows_), "BATproject");
    return out;
}

void Composer::multiRoundSorting()
{
    ensure_buffers();
    group_info_ = group_info_t();
    fmcs_ctx *ctx = GetContext();
    const auto t0 = std::chrono::steady_clock::now();
    const surrogate_t *in = nullptr;
    int cur = 0;
    uint32_t segments = 1;   // groups the next round sorts inside
    for (uint32_t c = 0; c < num_columns_; ++c) {
        Column *col = column_values_[c];
        const uint32_t bytes = col->GetWidth();
        const uint32_t bits = compose_params_.bitwidth ? compose_params_.bitwidth[c] : 8 * bytes;
        if (bytes == 1) throw std::runtime_error("fmcs: 8-bit columns cannot be sorted (src/mergesort.h:2926-2931)");
        const auto tr = std::chrono::steady_clock::now();
        uint32_t ng = 0;
        detail::check(fmcs_sort_round(ctx, col->GetColumn(), bytes, bits, d_order_, in, d_group_[cur], nullptr,
                                      num_rows_, &ng),
                      "multiRoundSorting");
        const double ms = ms_since(tr);
        if (c == 0) setting_.time_firstpass_sort = ms;
        setting_.time_multipass_sort += ms;
        if (c + 1 == num_columns_) {
            group_info_.ngroups = segments;
            group_info_.sum_group_size = (uint32_t)num_rows_;
        }
        segments = ng;
        ngroups_ = ng;
        in = d_group_[cur];
        final_group_ = cur;
        cur ^= 1;
    }
    setting_.time_orderGroupInfo = 0.0;   // group ids are fused into each round's timing
    (void)t0;
}

void Composer::hash_rounds(bool reordered)
{
    ensure_buffers();
    fmcs_ctx *ctx = GetContext();
    const surrogate_t *in = nullptr;
    int cur = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t c = 0; c < num_columns_; ++c) {
        Column *col = column_values_[c];
        const bool last = (c + 1 == num_columns_);
        uint32_t ng = 0;
        if (reordered) {
            detail::check(fmcs_hash_round(ctx, col->GetColumn(), col->GetWidth(), d_order_, in, d_group_[cur],
                                          num_rows_, last ? 1 : 0, &ng),
                          "multiRoundHashing_reordered");
        } else {
            detail::check(fmcs_hash_round_unordered(ctx, col->GetColumn(), col->GetWidth(), in, d_group_[cur],
                                                    num_rows_, &ng),
                          "multiRoundHashing_non_reordered");
        }
        ngroups_ = ng;
        in = d_group_[cur];
        final_group_ = cur;
        cur ^= 1;
    }
    if (!reordered && num_rows_) {
        // the order of a non-reordered grouping is the row order
        std::vector<surrogate_t> iota(num_rows_);
        for (uint64_t i = 0; i < num_rows_; ++i) iota[i] = (surrogate_t)i;
        cudaMemcpy(d_order_, iota.data(), num_rows_ * sizeof(surrogate_t), cudaMemcpyHostToDevice);
    }
    setting_.time_multipass_sort = ms_since(t0);
    group_info_.ngroups = ngroups_;
    group_info_.sum_group_size = (uint32_t)num_rows_;
}

void Composer::multiRoundHashing_reordered() { hash_rounds(true); }
void Composer::multiRoundHashing_partitioned_reordered() { hash_rounds(true); }
void Composer::multiRoundHashing_non_reordered() { hash_rounds(false); }

void ChainComposer::HashAllColumns()
{
    if (compose_params_.hash_type == 1)
        multiRoundHashing_reordered();
    else if (compose_params_.hash_type == 2)
        multiRoundHashing_partitioned_reordered();
    else
        multiRoundHashing_non_reordered();
}

}  // namespace multiAttrSort
