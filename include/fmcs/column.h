// fmcs/column.h -- Column / SpecialiedColumn<T>: one integer-coded column or
// massaged bank (reference: src/column.h:12-63, same class and method names).
//
// Storage is a raw T* that may point to host memory or to device memory (a
// column kept resident in HBM); every whole-column operation runs on the GPU
// through the C ABI.  ShiftLeftBatch and AssembleFromColumn keep the
// reference's semantics (src/column.h:105-180, 208-1060):
//   ShiftLeftBatch(n, k):          bank[i] <<= k                 (in place)
//   AssembleFromColumn(src, s, e, n, w):
//                                  bank[i] |= (src[i] >> (w - e)) & ((1 << (e-s+1)) - 1)
// A whole plan should use the fused stitch (StitchComposer::run_single_plan),
// which builds each bank in one pass instead of one pass per slice.
// The per-row accessors (SetValueAt, GetValueAt, ...) touch one element; on a
// device-resident column each is a small device copy.
#pragma once

#include <cstdint>

#include "../fmcs_capi.h"
#include "types.h"

namespace multiAttrSort {

/** The context the host classes use unless one is given explicitly: one per
 *  host thread, on the thread's current CUDA device (created on first use). */
FMCS_CXX_API fmcs_ctx *DefaultContext();

namespace detail {
FMCS_CXX_API void elem_read(const void *base, uint64_t idx, uint32_t bytes, void *out);
FMCS_CXX_API void elem_write(void *base, uint64_t idx, uint32_t bytes, const void *in);
FMCS_CXX_API void check(int rc, const char *what);   // throws std::runtime_error on failure
}  // namespace detail

template <class T>
class SpecialiedColumn;

class Column {
  public:
    virtual ~Column() {}
    virtual void *GetColumn() const = 0;
    virtual uint32_t GetWidth() const = 0;
    virtual void SetWidth(uint32_t w) = 0;
    virtual uint64_t GetCardinality() const = 0;
    virtual void SetCardinality(uint64_t card) = 0;

    virtual void SetValueAt(uint64_t val, uint64_t rowIdx) = 0;
    virtual void ShiftValueLeft(uint32_t nbits, uint64_t rowIdx) = 0;
    virtual void LogicalOr(uint64_t orValue, uint64_t rowIdx) = 0;
    virtual uint64_t GetValueAt(uint64_t rowIdx) const = 0;
    virtual uint64_t GetValPortion(uint64_t rowIdx, uint32_t start, uint32_t end) const = 0;
    virtual void ShiftLeftBatch(uint64_t num_rows, uint32_t nbits) = 0;
    virtual void AssembleFromColumn(SpecialiedColumn<uint8_t> *fromColumn, uint32_t start, uint32_t end,
                                    uint64_t num_rows, uint32_t originWidth) = 0;
    virtual void AssembleFromColumn(SpecialiedColumn<uint16_t> *fromColumn, uint32_t start, uint32_t end,
                                    uint64_t num_rows, uint32_t originWidth) = 0;
    virtual void AssembleFromColumn(SpecialiedColumn<uint32_t> *fromColumn, uint32_t start, uint32_t end,
                                    uint64_t num_rows, uint32_t originWidth) = 0;
    virtual void AssembleFromColumn(SpecialiedColumn<uint64_t> *fromColumn, uint32_t start, uint32_t end,
                                    uint64_t num_rows, uint32_t originWidth) = 0;
};

template <class T>
class SpecialiedColumn : public Column {
  public:
    SpecialiedColumn() : values_(nullptr), width_(sizeof(T)), cardinality_(0) {}
    ~SpecialiedColumn() override {}

    void *GetColumn() const override { return (void *)values_; }
    void SetColumn(T *values) { values_ = values; }
    uint32_t GetWidth() const override { return width_; }
    void SetWidth(uint32_t w) override { width_ = w; }
    uint64_t GetCardinality() const override { return cardinality_; }
    void SetCardinality(uint64_t card) override { cardinality_ = card; }

    void SetValueAt(uint64_t val, uint64_t rowIdx) override
    {
        T v = (T)val;
        detail::elem_write(values_, rowIdx, sizeof(T), &v);
    }
    void ShiftValueLeft(uint32_t nbits, uint64_t rowIdx) override
    {
        T v;
        detail::elem_read(values_, rowIdx, sizeof(T), &v);
        v = (T)(v << nbits);
        detail::elem_write(values_, rowIdx, sizeof(T), &v);
    }
    void LogicalOr(uint64_t orValue, uint64_t rowIdx) override
    {
        T v;
        detail::elem_read(values_, rowIdx, sizeof(T), &v);
        v = (T)(v | orValue);
        detail::elem_write(values_, rowIdx, sizeof(T), &v);
    }
    uint64_t GetValueAt(uint64_t rowIdx) const override
    {
        T v;
        detail::elem_read(values_, rowIdx, sizeof(T), &v);
        return (uint64_t)v;
    }
    // bits [start, end] counted 1-based from the LSB (reference: src/column.h:196-206)
    uint64_t GetValPortion(uint64_t rowIdx, uint32_t start, uint32_t end) const override
    {
        uint64_t v = GetValueAt(rowIdx) >> (start - 1);
        const uint32_t w = end - start + 1;
        return w >= 64 ? v : (v & ((1ull << w) - 1));
    }
    void ShiftLeftBatch(uint64_t num_rows, uint32_t nbits) override
    {
        detail::check(fmcs_shift_left(DefaultContext(), values_, sizeof(T), num_rows, nbits), "ShiftLeftBatch");
    }
    void AssembleFromColumn(SpecialiedColumn<uint8_t> *from, uint32_t start, uint32_t end, uint64_t num_rows,
                            uint32_t originWidth) override
    {
        assemble(from->GetColumn(), 1, start, end, num_rows, originWidth);
    }
    void AssembleFromColumn(SpecialiedColumn<uint16_t> *from, uint32_t start, uint32_t end, uint64_t num_rows,
                            uint32_t originWidth) override
    {
        assemble(from->GetColumn(), 2, start, end, num_rows, originWidth);
    }
    void AssembleFromColumn(SpecialiedColumn<uint32_t> *from, uint32_t start, uint32_t end, uint64_t num_rows,
                            uint32_t originWidth) override
    {
        assemble(from->GetColumn(), 4, start, end, num_rows, originWidth);
    }
    void AssembleFromColumn(SpecialiedColumn<uint64_t> *from, uint32_t start, uint32_t end, uint64_t num_rows,
                            uint32_t originWidth) override
    {
        assemble(from->GetColumn(), 8, start, end, num_rows, originWidth);
    }

  private:
    void assemble(const void *src, uint32_t src_bytes, uint32_t start, uint32_t end, uint64_t n, uint32_t w)
    {
        fmcs_slice s{src, src_bytes, w, start, end};
        detail::check(fmcs_assemble(DefaultContext(), values_, sizeof(T), n, &s), "AssembleFromColumn");
    }

    T *values_;
    uint32_t width_;         // bytes per value
    uint64_t cardinality_;   // number of distinct values (statistics for the cost model)
};

}  // namespace multiAttrSort
