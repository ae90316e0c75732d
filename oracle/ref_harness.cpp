/*
 * ref_harness.cpp -- drives the REFERENCE implementation (FastMultiColSort's
 * own composer, bit stitching and hash grouping code) so that its outputs can
 * pin the oracle and serve as the timed CPU baseline.  TEST INFRASTRUCTURE
 * ONLY.  The reference sources are #included at build time from the
 * reference tree given to oracle/Makefile (FMCS_REF); nothing of them is
 * copied into this repository.  The product never links this file.
 *
 * Why a harness: the reference frees its outputs inside multiRoundSorting
 * (src/composer.cpp:132-134), so the harness calls the per-round entry points
 * itself.  Composer members are public (`//protected:` at src/composer.h:50).
 *
 * Quirks of the reference that the harness works around (documented in the
 * design notes):
 *   - multiRoundHashing_reordered passes `histogram` by value, so rounds after
 *     the first get NULL (src/composer.cpp:150-193, 868); the harness passes a
 *     buffer of n entries to every round.
 *   - hashByGroup_* prints a line per round to std::cout; the harness mutes
 *     std::cout while the reference runs.
 */
#include "composer.cpp"
#include "chain_composer.cpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

using namespace multiAttrSort;

namespace {

struct MuteCout {
    MuteCout() { std::cout.setstate(std::ios_base::failbit); }
    ~MuteCout() { std::cout.clear(); }
};

Column *make_column(uint32_t bytes, uint64_t n, const void *init)
{
    size_t sz = (size_t)(n ? n : 1) * bytes + 64;
    void *mem = malloc_aligned(sz);
    if (!mem) return nullptr;
    memset(mem, 0, sz);
    if (init && n) memcpy(mem, init, (size_t)n * bytes);
    switch (bytes) {
    case 1: { auto *c = new SpecialiedColumn<uint8_t>(); c->SetColumn((uint8_t *)mem); c->SetWidth(1); return c; }
    case 2: { auto *c = new SpecialiedColumn<uint16_t>(); c->SetColumn((uint16_t *)mem); c->SetWidth(2); return c; }
    case 4: { auto *c = new SpecialiedColumn<uint32_t>(); c->SetColumn((uint32_t *)mem); c->SetWidth(4); return c; }
    case 8: { auto *c = new SpecialiedColumn<uint64_t>(); c->SetColumn((uint64_t *)mem); c->SetWidth(8); return c; }
    }
    free(mem);
    return nullptr;
}

void free_column(Column *c)
{
    if (!c) return;
    free(c->GetColumn());
    delete c;
}

/* The reference's stitch loop, src/stitch_composer.cpp:655-703: shift the bank
 * for every slice but the first, then OR the slice in. */
void assemble(Column *bank, Column *src, uint32_t start, uint32_t end, uint64_t n, uint32_t bw)
{
    switch (src->GetWidth()) {
    case 1: bank->AssembleFromColumn(reinterpret_cast<SpecialiedColumn<uint8_t> *>(src), start, end, n, bw); break;
    case 2: bank->AssembleFromColumn(reinterpret_cast<SpecialiedColumn<uint16_t> *>(src), start, end, n, bw); break;
    case 4: bank->AssembleFromColumn(reinterpret_cast<SpecialiedColumn<uint32_t> *>(src), start, end, n, bw); break;
    case 8: bank->AssembleFromColumn(reinterpret_cast<SpecialiedColumn<uint64_t> *>(src), start, end, n, bw); break;
    }
}

/* Slice records in the shape of construct_entry_t (src/types.h:42-46), built by
 * the same walk as src/stitch_composer.cpp:568-612 with column order 0..k-1. */
bool build_records(const uint32_t *bw, uint32_t ncols, const uint32_t *split, uint32_t nbanks,
                   std::vector<std::vector<construct_entry_t>> &out)
{
    uint32_t so = 0, sn = 0;
    for (uint32_t c = 0; c < ncols; ++c) so += bw[c];
    for (uint32_t b = 0; b < nbanks; ++b) { if (!split[b] || split[b] > 64) return false; sn += split[b]; }
    if (!ncols || !nbanks || so != sn) return false;
    out.assign(nbanks, {});
    uint32_t oc = 0, nb = 0, start = 1, ol = bw[0], nl = split[0];
    while (nb < nbanks) {
        uint32_t take = ol < nl ? ol : nl;
        construct_entry_t e;
        e.finalIdx = oc;
        e.start = start;
        e.end = start + take - 1;
        out[nb].push_back(e);
        start += take;
        ol -= take;
        nl -= take;
        if (!ol) { oc++; if (oc < ncols) ol = bw[oc]; start = 1; }
        if (!nl) { nb++; if (nb < nbanks) nl = split[nb]; }
    }
    return true;
}

uint32_t bank_bytes_for(uint32_t bits, bool hash_path)
{
    if (hash_path && bits <= 8) return 1;   /* src/stitch_composer.cpp:883-890 */
    if (bits <= 16) return 2;               /* :622-650 */
    if (bits <= 32) return 4;
    return 8;
}

ChainComposer *make_composer(uint64_t n, uint32_t nbanks, Column **banks, bool *asc, uint32_t *bits)
{
    setting_t setting;
    setting.nthreads = 1;
    setting.intrinType = IntrinsicsType::AVX;
    compose_params_t params;
    params.column_asc_desc = asc;
    params.bitwidth = bits;
    params.hash_type = 1;
    return new ChainComposer(setting, nbanks, n, params, banks);
}

template <class T>
void sort_round(ChainComposer *cc, uint32_t *out_group, Column *bank, uint32_t *order,
                uint32_t *in_group, uint32_t bits, bool last)
{
    cc->sortByGroup<T>(out_group, (T *)bank->GetColumn(), order, in_group, true, bits, last);
}

template <class T>
void hash_round(ChainComposer *cc, uint32_t *out_group, uint32_t *out_order, Column *bank,
                uint32_t *in_order, uint32_t *in_group, bool last, Hash_t *h,
                uint32_t *idx, uint32_t *hist)
{
    cc->hashByGroup_reordered<T>(out_group, out_order, (T *)bank->GetColumn(), in_order, in_group,
                                 last, h, idx, hist);
}

}  // namespace

extern "C" {

/* Stitch one bank with the reference's ShiftLeftBatch/AssembleFromColumn. */
int ref_stitch(const void *const *srcs, const uint32_t *src_bytes, const uint32_t *src_bits,
               const uint32_t *starts, const uint32_t *ends, uint32_t nslices,
               void *bank_out, uint32_t bank_bytes, uint64_t n)
{
    Column *bank = make_column(bank_bytes, n, nullptr);
    if (!bank) return -2;
    for (uint32_t s = 0; s < nslices; ++s) {
        Column *src = make_column(src_bytes[s], n, srcs[s]);
        if (!src) { free_column(bank); return -2; }
        if (s) bank->ShiftLeftBatch(n, ends[s] - starts[s] + 1);
        assemble(bank, src, starts[s], ends[s], n, src_bits[s]);
        free_column(src);
    }
    memcpy(bank_out, bank->GetColumn(), (size_t)n * bank_bytes);
    free_column(bank);
    return 0;
}

/* Whole sort plan: stitch (reference code) then one sortByGroup per bank.
 * final_groups != 0 computes the last round's group vector as well (the
 * reference skips it, src/composer.cpp:1388-1390); 0 times the reference's
 * own run exactly.  *seconds gets the steady_clock time of stitch + rounds. */
int ref_run_plan_sort(const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                      uint32_t ncols, const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, int final_groups,
                      double *seconds)
{
    std::vector<std::vector<construct_entry_t>> rec;
    if (!build_records(bw, ncols, split, nbanks, rec) || n < 1 || n > 0xFFFFFFFFull) return -1;
    for (uint32_t c = 0; c < ncols; ++c) if (col_bytes[c] == 1) return -1;  /* :681-687 */
    std::vector<Column *> src(ncols), banks(nbanks);
    for (uint32_t c = 0; c < ncols; ++c) src[c] = make_column(col_bytes[c], n, cols[c]);
    std::vector<uint8_t> asc(nbanks, 1);
    std::vector<uint32_t> bits(split, split + nbanks);
    uint32_t *order = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *ga = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *gb = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    MuteCout mute;
    auto t0 = std::chrono::steady_clock::now();
    for (uint32_t b = 0; b < nbanks; ++b) {
        banks[b] = make_column(bank_bytes_for(split[b], false), n, nullptr);
        for (size_t k = 0; k < rec[b].size(); ++k) {
            const construct_entry_t &e = rec[b][k];
            if (k) banks[b]->ShiftLeftBatch(n, e.end - e.start + 1);
            assemble(banks[b], src[e.finalIdx], e.start, e.end, n, bw[e.finalIdx]);
        }
    }
    ChainComposer *cc = make_composer(n, nbanks, banks.data(), (bool *)asc.data(), bits.data());
    for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    uint32_t *in = nullptr, *out = ga;
    for (uint32_t b = 0; b < nbanks; ++b) {
        bool last = (b + 1 == nbanks) && !final_groups;
        switch (banks[b]->GetWidth()) {
        case 2: sort_round<uint16_t>(cc, out, banks[b], order, in, split[b], last); break;
        case 4: sort_round<uint32_t>(cc, out, banks[b], order, in, split[b], last); break;
        case 8: sort_round<uint64_t>(cc, out, banks[b], order, in, split[b], last); break;
        }
        in = out;
        out = (out == ga) ? gb : ga;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (order_out) memcpy(order_out, order, n * sizeof(uint32_t));
    if (group_out && final_groups) memcpy(group_out, in, n * sizeof(uint32_t));
    cc->column_values_ = nullptr;
    delete cc;
    for (auto *c : banks) free_column(c);
    for (auto *c : src) free_column(c);
    free(order); free(ga); free(gb);
    return 0;
}

/* One sort round on an existing bank (reference sortByGroup<T>).  bank is not
 * modified (round 0 sorts a copy).  sorted_keys may be NULL. */
int ref_sort_round(const void *bank_in, uint32_t bank_bytes, uint32_t bits, uint32_t *order,
                   const uint32_t *in_group, uint32_t *out_group, uint64_t n)
{
    if (bank_bytes == 1 || n < 1) return -1;
    Column *bank = make_column(bank_bytes, n, bank_in);
    std::vector<uint8_t> asc(1, 1);
    std::vector<uint32_t> bw(1, bits);
    Column *cols[1] = {bank};
    uint32_t *ord = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *ig = nullptr;
    if (in_group) {
        ig = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
        memcpy(ig, in_group, n * sizeof(uint32_t));
        memcpy(ord, order, n * sizeof(uint32_t));
    } else {
        for (uint64_t i = 0; i < n; ++i) ord[i] = (uint32_t)i;
    }
    MuteCout mute;
    ChainComposer *cc = make_composer(n, 1, cols, (bool *)asc.data(), bw.data());
    switch (bank_bytes) {
    case 2: sort_round<uint16_t>(cc, out_group, bank, ord, ig, bits, out_group == nullptr); break;
    case 4: sort_round<uint32_t>(cc, out_group, bank, ord, ig, bits, out_group == nullptr); break;
    case 8: sort_round<uint64_t>(cc, out_group, bank, ord, ig, bits, out_group == nullptr); break;
    }
    memcpy(order, ord, n * sizeof(uint32_t));
    cc->column_values_ = nullptr;
    delete cc;
    free_column(bank);
    free(ord);
    free(ig);
    return 0;
}

/* Whole hash plan: stitch (reference code, u8 banks allowed) then one
 * hashByGroup_reordered per bank.  order_out gets the last round's input
 * order, group_out the last round's intermediate_group_idx. */
int ref_run_plan_hash(const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                      uint32_t ncols, const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, double *seconds)
{
    std::vector<std::vector<construct_entry_t>> rec;
    if (!build_records(bw, ncols, split, nbanks, rec) || n < 1 || n > 0xFFFFFFFFull) return -1;
    std::vector<Column *> src(ncols), banks(nbanks);
    for (uint32_t c = 0; c < ncols; ++c) src[c] = make_column(col_bytes[c], n, cols[c]);
    std::vector<uint8_t> asc(nbanks, 1);
    std::vector<uint32_t> bits(split, split + nbanks);
    uint32_t *io = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *oo = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *ga = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *gb = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *idx = (uint32_t *)malloc_aligned(n * sizeof(uint32_t));
    uint32_t *hist = (uint32_t *)malloc_aligned((n + 1) * sizeof(uint32_t));
    MuteCout mute;
    auto t0 = std::chrono::steady_clock::now();
    for (uint32_t b = 0; b < nbanks; ++b) {
        banks[b] = make_column(bank_bytes_for(split[b], true), n, nullptr);
        for (size_t k = 0; k < rec[b].size(); ++k) {
            const construct_entry_t &e = rec[b][k];
            if (k) banks[b]->ShiftLeftBatch(n, e.end - e.start + 1);
            assemble(banks[b], src[e.finalIdx], e.start, e.end, n, bw[e.finalIdx]);
        }
    }
    ChainComposer *cc = make_composer(n, nbanks, banks.data(), (bool *)asc.data(), bits.data());
    Hash_t *h = (Hash_t *)malloc_aligned(sizeof(Hash_t));
    cc->createHashTable(h);
    for (uint64_t i = 0; i < n; ++i) { io[i] = (uint32_t)i; oo[i] = (uint32_t)i; }
    uint32_t *in = nullptr, *out = ga;
    for (uint32_t b = 0; b < nbanks; ++b) {
        bool last = (b + 1 == nbanks);
        /* round 0 allocates its own histogram inside the reference */
        uint32_t *hp = in ? hist : nullptr;
        switch (banks[b]->GetWidth()) {
        case 1: hash_round<uint8_t>(cc, out, oo, banks[b], io, in, last, h, idx, hp); break;
        case 2: hash_round<uint16_t>(cc, out, oo, banks[b], io, in, last, h, idx, hp); break;
        case 4: hash_round<uint32_t>(cc, out, oo, banks[b], io, in, last, h, idx, hp); break;
        case 8: hash_round<uint64_t>(cc, out, oo, banks[b], io, in, last, h, idx, hp); break;
        }
        if (!last) {
            uint32_t *t = in ? in : gb;
            in = out;
            out = t;
            std::swap(io, oo);
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (order_out) memcpy(order_out, io, n * sizeof(uint32_t));
    if (group_out) memcpy(group_out, idx, n * sizeof(uint32_t));
    free(h->Link);
    free(h);
    cc->column_values_ = nullptr;
    delete cc;
    for (auto *c : banks) free_column(c);
    for (auto *c : src) free_column(c);
    free(io); free(oo); free(ga); free(gb); free(idx); free(hist);
    return 0;
}

}  // extern "C"
