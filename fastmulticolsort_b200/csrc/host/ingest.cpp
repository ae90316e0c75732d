// ingest.cpp -- the reference's text dataset format, read and written on the host.
//
// Reference: DataGenerator::ReadFromFile / ReadFromFile_tpch / ReadValues and
// GenAndSaveAsFile (src/generator.h:43-136, 138-227).  A dataset file holds
// unsigned decimal values separated by white space (one per line as
// written), column after column: all rows of column 0, then column 1, ...
// The TPC-H variant starts with two numbers, the row count and the column
// count.  Each column is stored in the width its declared bit width maps to
// (src/generator.h:88-94): up to 16 bits u16, up to 32 bits u32, else u64; its
// cardinality is its number of distinct values (ReadValues' std::set).
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../../include/fmcs_capi.h"

namespace {

// Buffered reader of unsigned decimal numbers separated by white space.
class NumberReader {
  public:
    explicit NumberReader(FILE *f) : f_(f), buf_(1 << 20) {}
    // 1: a number in *v; 0: end of file; -1: malformed input or overflow.
    int next(uint64_t *v)
    {
        int c;
        do {
            c = get();
        } while (c == ' ' || c == '\n' || c == '\r' || c == '\t');
        if (c < 0) return 0;
        if (c < '0' || c > '9') return -1;
        uint64_t x = 0;
        while (c >= '0' && c <= '9') {
            const uint64_t d = (uint64_t)(c - '0');
            if (x > (UINT64_MAX - d) / 10) return -1;
            x = x * 10 + d;
            c = get();
        }
        if (c >= 0 && !(c == ' ' || c == '\n' || c == '\r' || c == '\t')) return -1;
        *v = x;
        return 1;
    }

  private:
    int get()
    {
        if (pos_ == len_) {
            len_ = fread(buf_.data(), 1, buf_.size(), f_);
            pos_ = 0;
            if (len_ == 0) return -1;
        }
        return (unsigned char)buf_[pos_++];
    }
    FILE *f_;
    std::vector<char> buf_;
    size_t pos_ = 0, len_ = 0;
};

template <typename T>
uint64_t distinct_count(const T *v, uint64_t n)
{
    std::vector<T> s(v, v + n);
    std::sort(s.begin(), s.end());
    return (uint64_t)(std::unique(s.begin(), s.end()) - s.begin());
}

}  // namespace

extern "C" uint32_t fmcs_storage_bytes(uint32_t bw)
{
    return bw == 0 || bw > 64 ? 0u : (bw <= 16 ? 2u : (bw <= 32 ? 4u : 8u));
}

extern "C" int fmcs_text_header(const char *path, uint64_t *nrows, uint32_t *ncols)
{
    if (!path || !nrows || !ncols) return FMCS_E_INVAL;
    FILE *f = fopen(path, "rb");
    if (!f) return FMCS_E_INVAL;
    NumberReader in(f);
    uint64_t a = 0, b = 0;
    const int ok = in.next(&a) == 1 && in.next(&b) == 1 && b <= 0xFFFFFFFFull;
    fclose(f);
    if (!ok) return FMCS_E_INVAL;
    *nrows = a;
    *ncols = (uint32_t)b;
    return FMCS_OK;
}

extern "C" int fmcs_read_columns_text(const char *path, int has_header, uint32_t ncols, const uint32_t *bw,
                                      uint64_t nrows, void *const *cols_out, uint64_t *cardinality_out)
{
    if (!path || !bw || !cols_out || ncols == 0) return FMCS_E_INVAL;
    for (uint32_t c = 0; c < ncols; ++c)
        if (fmcs_storage_bytes(bw[c]) == 0 || (nrows && !cols_out[c])) return FMCS_E_INVAL;
    FILE *f = fopen(path, "rb");
    if (!f) return FMCS_E_INVAL;
    NumberReader in(f);
    int rc = FMCS_OK;
    uint64_t v;
    if (has_header) {
        uint64_t hn = 0, hc = 0;
        if (in.next(&hn) != 1 || in.next(&hc) != 1 || hn != nrows) rc = FMCS_E_INVAL;
        (void)hc;   // the reference reads and ignores the stored column count
    }
    for (uint32_t c = 0; c < ncols && rc == FMCS_OK; ++c) {
        const uint32_t bytes = fmcs_storage_bytes(bw[c]);
        const uint64_t vmax = bytes == 8 ? UINT64_MAX : ((1ull << (8 * bytes)) - 1);
        for (uint64_t i = 0; i < nrows; ++i) {
            if (in.next(&v) != 1 || v > vmax) {
                rc = FMCS_E_INVAL;
                break;
            }
            switch (bytes) {
            case 2: ((uint16_t *)cols_out[c])[i] = (uint16_t)v; break;
            case 4: ((uint32_t *)cols_out[c])[i] = (uint32_t)v; break;
            default: ((uint64_t *)cols_out[c])[i] = v; break;
            }
        }
    }
    fclose(f);
    if (rc != FMCS_OK || !cardinality_out) return rc;
    for (uint32_t c = 0; c < ncols; ++c) {
        switch (fmcs_storage_bytes(bw[c])) {
        case 2: cardinality_out[c] = distinct_count((const uint16_t *)cols_out[c], nrows); break;
        case 4: cardinality_out[c] = distinct_count((const uint32_t *)cols_out[c], nrows); break;
        default: cardinality_out[c] = distinct_count((const uint64_t *)cols_out[c], nrows); break;
        }
    }
    return FMCS_OK;
}

extern "C" int fmcs_write_columns_text(const char *path, int with_header, uint32_t ncols, uint64_t nrows,
                                       const void *const *cols, const uint32_t *col_bytes)
{
    if (!path || !cols || !col_bytes || ncols == 0) return FMCS_E_INVAL;
    for (uint32_t c = 0; c < ncols; ++c)
        if (!(col_bytes[c] == 2 || col_bytes[c] == 4 || col_bytes[c] == 8) || (nrows && !cols[c]))
            return FMCS_E_INVAL;
    FILE *f = fopen(path, "wb");
    if (!f) return FMCS_E_INVAL;
    std::vector<char> out;
    out.reserve(1 << 21);
    char num[24];
    auto flush = [&]() {
        if (!out.empty() && fwrite(out.data(), 1, out.size(), f) != out.size()) return false;
        out.clear();
        return true;
    };
    bool ok = true;
    if (with_header) ok = fprintf(f, "%llu\n%u\n", (unsigned long long)nrows, ncols) > 0;
    for (uint32_t c = 0; c < ncols && ok; ++c) {
        for (uint64_t i = 0; i < nrows && ok; ++i) {
            uint64_t v;
            switch (col_bytes[c]) {
            case 2: v = ((const uint16_t *)cols[c])[i]; break;
            case 4: v = ((const uint32_t *)cols[c])[i]; break;
            default: v = ((const uint64_t *)cols[c])[i]; break;
            }
            int k = 0;
            do {
                num[k++] = (char)('0' + v % 10);
                v /= 10;
            } while (v);
            while (k) out.push_back(num[--k]);
            out.push_back('\n');
            if (out.size() >= (1 << 20)) ok = flush();
        }
    }
    if (ok) ok = flush();
    if (fclose(f) != 0) ok = false;
    return ok ? FMCS_OK : FMCS_E_INVAL;
}
