/*
 * fmcs_oracle.c -- CPU restatement of FastMultiColSort's multi-column sort
 * path.  TEST INFRASTRUCTURE ONLY: the parity oracle of the CUDA path.  The shipped
 * library never links or calls it.  Every function cites the reference code
 * it restates (paths are relative to the reference project root).
 *
 * The restatement is plain scalar C.  Sorting is a stable LSD radix sort,
 * which gives the reference's results with ties canonicalised to ascending
 * oid (the reference's AVX merge sort is not stable; src/composer.cpp:490-556).
 */
#include "fmcs_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* typed access                                                              */
/* ------------------------------------------------------------------------ */
static inline uint64_t ld(const void *p, uint32_t bytes, uint64_t i)
{
    switch (bytes) {
    case 1: return ((const uint8_t *)p)[i];
    case 2: return ((const uint16_t *)p)[i];
    case 4: return ((const uint32_t *)p)[i];
    default: return ((const uint64_t *)p)[i];
    }
}

static inline void st(void *p, uint32_t bytes, uint64_t i, uint64_t v)
{
    switch (bytes) {
    case 1: ((uint8_t *)p)[i] = (uint8_t)v; break;
    case 2: ((uint16_t *)p)[i] = (uint16_t)v; break;
    case 4: ((uint32_t *)p)[i] = (uint32_t)v; break;
    default: ((uint64_t *)p)[i] = v; break;
    }
}

static inline int valid_bytes(uint32_t b) { return b == 1 || b == 2 || b == 4 || b == 8; }

/* ------------------------------------------------------------------------ */
/* plan records, src/stitch_composer.cpp:568-612                             */
/* ------------------------------------------------------------------------ */
int orc_plan_records(const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                     const uint32_t *split, uint32_t nbanks,
                     orc_record *rec, uint32_t *nrec)
{
    uint32_t total_old = 0, total_new = 0;
    for (uint32_t c = 0; c < ncols; ++c) total_old += bw[c];
    for (uint32_t b = 0; b < nbanks; ++b) {
        if (split[b] == 0 || split[b] > 64) return -1;
        total_new += split[b];
        nrec[b] = 0;
    }
    if (ncols == 0 || nbanks == 0 || total_old != total_new) return -1;

    /* Walk the old columns (in col_order) and the new banks together; each
     * step consumes min(remaining old bits, remaining bank bits). */
    uint32_t oc = 0, nb = 0, start = 1, nr = 0;
    uint32_t old_left = bw[col_order[0]], new_left = split[0];
    while (nb < nbanks) {
        uint32_t take = old_left < new_left ? old_left : new_left;
        rec[nr].final_idx = col_order[oc];
        rec[nr].start = start;
        rec[nr].end = start + take - 1;
        nr++;
        nrec[nb]++;
        start += take;
        old_left -= take;
        new_left -= take;
        if (old_left == 0) {
            oc++;
            if (oc < ncols) old_left = bw[col_order[oc]];
            start = 1;
        }
        if (new_left == 0) {
            nb++;
            if (nb < nbanks) new_left = split[nb];
        }
    }
    return (int)nr;
}

/* src/stitch_composer.cpp:622-650 (sort) and :879-912 (hash, allows u8). */
uint32_t orc_bank_bytes(uint32_t bits, int hash_path)
{
    if (hash_path && bits <= 8) return 1;
    if (bits <= 16) return 2;
    if (bits <= 32) return 4;
    return 8;
}

/* ------------------------------------------------------------------------ */
/* stitch, src/column.h:105-180 (ShiftLeftBatch), 208-1060 (AssembleFromColumn)
 * bank := (bank << width) | ((src >> (src_bits - end)) & mask), the first slice
 * unshifted (src/stitch_composer.cpp:664-703).  A 64-bit-wide slice uses a
 * full mask; the reference computes (1ULL<<64)-1 there, which x86 evaluates to
 * 0, so such slices are outside the parity domain.                           */
/* ------------------------------------------------------------------------ */
int orc_stitch(const orc_slice *sl, uint32_t ns, void *bank, uint32_t bank_bytes, uint64_t n)
{
    if (!valid_bytes(bank_bytes) || ns == 0) return -1;
    for (uint32_t s = 0; s < ns; ++s) {
        if (!valid_bytes(sl[s].src_bytes) || sl[s].start < 1 || sl[s].end < sl[s].start ||
            sl[s].end > sl[s].src_bits || sl[s].src_bits > 64)
            return -1;
    }
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t acc = 0;
        for (uint32_t s = 0; s < ns; ++s) {
            uint32_t w = sl[s].end - sl[s].start + 1;
            uint64_t mask = (w >= 64) ? ~0ULL : ((1ULL << w) - 1);
            uint64_t v = ld(sl[s].src, sl[s].src_bytes, i) >> (sl[s].src_bits - sl[s].end);
            v &= mask;
            acc = (s == 0) ? v : (((w >= 64) ? 0 : (acc << w)) | v);
        }
        st(bank, bank_bytes, i, acc);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* stable LSD radix sort of (key, payload) pairs                             */
/* ------------------------------------------------------------------------ */
static void lsd_sort(uint64_t *key, uint32_t *val, uint64_t n, uint32_t key_bytes,
                     uint64_t *ktmp, uint32_t *vtmp)
{
    size_t cnt[256];
    uint64_t *ka = key, *kb = ktmp;
    uint32_t *va = val, *vb = vtmp;
    for (uint32_t pass = 0; pass < key_bytes; ++pass) {
        uint32_t sh = pass * 8;
        memset(cnt, 0, sizeof(cnt));
        for (uint64_t i = 0; i < n; ++i) cnt[(ka[i] >> sh) & 0xFF]++;
        /* a pass where every key has the same digit is the identity */
        int trivial = 0;
        for (int d = 0; d < 256; ++d) if (cnt[d] == n) trivial = 1;
        if (trivial) continue;
        size_t sum = 0;
        for (int d = 0; d < 256; ++d) { size_t c = cnt[d]; cnt[d] = sum; sum += c; }
        for (uint64_t i = 0; i < n; ++i) {
            size_t p = cnt[(ka[i] >> sh) & 0xFF]++;
            kb[p] = ka[i];
            vb[p] = va[i];
        }
        uint64_t *kt = ka; ka = kb; kb = kt;
        uint32_t *vt = va; va = vb; vb = vt;
    }
    if (ka != key) {
        memcpy(key, ka, n * sizeof(uint64_t));
        memcpy(val, va, n * sizeof(uint32_t));
    }
}

/* ------------------------------------------------------------------------ */
/* one sort round, src/composer.cpp:1222-1408                                */
/* ------------------------------------------------------------------------ */
int orc_sort_round(const void *bank, uint32_t bank_bytes, uint32_t *order,
                   const uint32_t *in_group, uint32_t *out_group,
                   void *sorted_keys, uint64_t n, uint32_t *ngroups)
{
    if (!valid_bytes(bank_bytes)) return -1;
    if (ngroups) *ngroups = 0;
    if (n == 0) return 0;
    uint64_t *key = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *ktmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint32_t *vtmp = (uint32_t *)malloc(n * sizeof(uint32_t));
    if (!key || !ktmp || !vtmp) { free(key); free(ktmp); free(vtmp); return -2; }

    if (in_group == NULL) {
        /* round 0: order starts as iota, src/composer.cpp:60-63 */
        for (uint64_t i = 0; i < n; ++i) { order[i] = (uint32_t)i; key[i] = ld(bank, bank_bytes, i); }
        lsd_sort(key, order, n, bank_bytes, ktmp, vtmp);
    } else {
        /* BATproject, src/composer.cpp:608-628 */
        for (uint64_t i = 0; i < n; ++i) key[i] = ld(bank, bank_bytes, order[i]);
        /* Stable sort inside every run of equal in_group (:1280-1335):
         * sort (key, position) stably by key, then stably by run id. */
        uint32_t *pos = (uint32_t *)malloc(n * sizeof(uint32_t));
        uint32_t *run = (uint32_t *)malloc(n * sizeof(uint32_t));
        size_t *rstart = (size_t *)malloc((n + 1) * sizeof(size_t));
        uint32_t *neworder = (uint32_t *)malloc(n * sizeof(uint32_t));
        if (!pos || !run || !rstart || !neworder) {
            free(pos); free(run); free(rstart); free(neworder);
            free(key); free(ktmp); free(vtmp); return -2;
        }
        uint32_t r = 0;
        rstart[0] = 0;
        for (uint64_t i = 0; i < n; ++i) {
            if (i > 0 && in_group[i] != in_group[i - 1]) { r++; rstart[r] = i; }
            run[i] = r;
            pos[i] = (uint32_t)i;
        }
        lsd_sort(key, pos, n, bank_bytes, ktmp, vtmp);
        /* stable scatter by run id: run r occupies [rstart[r], rstart[r+1]) */
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t p = pos[i];
            size_t dst = rstart[run[p]]++;
            neworder[dst] = order[p];
            ktmp[dst] = key[i];
        }
        memcpy(order, neworder, n * sizeof(uint32_t));
        memcpy(key, ktmp, n * sizeof(uint64_t));
        free(pos); free(run); free(rstart); free(neworder);
    }

    if (sorted_keys)
        for (uint64_t i = 0; i < n; ++i) st(sorted_keys, bank_bytes, i, key[i]);

    /* extractGroupInfo, src/composer.cpp:630-678 */
    if (out_group) {
        uint32_t g = 0;
        out_group[0] = 0;
        for (uint64_t i = 1; i < n; ++i) {
            g += (key[i] != key[i - 1]) || (in_group && in_group[i] != in_group[i - 1]);
            out_group[i] = g;
        }
        if (ngroups) *ngroups = g + 1;
    }
    free(key); free(ktmp); free(vtmp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* one hash round, src/composer.cpp:814-976                                  */
/* ------------------------------------------------------------------------ */
static inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

int orc_hash_round(const void *bank, uint32_t bank_bytes, uint32_t *order,
                   const uint32_t *in_group, uint32_t *out_group,
                   uint32_t *group_idx, uint64_t n, int last_round,
                   uint32_t *ngroups)
{
    if (!valid_bytes(bank_bytes)) return -1;
    if (ngroups) *ngroups = 0;
    if (n == 0) return 0;
    if (!last_round && !out_group) return -1;
    uint64_t *key = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t tsize = 16;
    while (tsize < 2 * n) tsize <<= 1;
    uint32_t *slot_row = (uint32_t *)malloc(tsize * sizeof(uint32_t));   /* position of first row */
    uint32_t *hist = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
    uint32_t *neworder = (uint32_t *)malloc(n * sizeof(uint32_t));
    if (!key || !slot_row || !hist || !neworder) {
        free(key); free(slot_row); free(hist); free(neworder); return -2;
    }
    if (in_group == NULL) {
        for (uint64_t i = 0; i < n; ++i) { order[i] = (uint32_t)i; key[i] = ld(bank, bank_bytes, i); }
    } else {
        for (uint64_t i = 0; i < n; ++i) key[i] = ld(bank, bank_bytes, order[i]);   /* BATproject */
    }

    uint32_t next_id = 0;   /* startGrpIdx */
    uint64_t start = 0;
    while (start < n) {
        uint64_t end = start + 1;
        if (in_group) while (end < n && in_group[end] == in_group[start]) end++;
        else end = n;
        uint64_t len = end - start;
        /* first-appearance numbering, Hashing::subgroup_range (hashing.h:289-385) */
        uint64_t ts = 16;
        while (ts < 2 * len) ts <<= 1;
        memset(slot_row, 0xFF, ts * sizeof(uint32_t));
        uint32_t base = next_id;
        for (uint64_t i = start; i < end; ++i) {
            uint64_t h = mix64(key[i]) & (ts - 1);
            for (;;) {
                uint32_t r = slot_row[h];
                if (r == 0xFFFFFFFFu) {
                    slot_row[h] = (uint32_t)i;
                    group_idx[i] = next_id++;
                    break;
                }
                if (key[r] == key[i]) { group_idx[i] = group_idx[r]; break; }
                h = (h + 1) & (ts - 1);
            }
        }
        uint32_t ng = next_id - base;
        /* stable counting scatter, Partition::histogram_based_reordering
         * (partition.h:44-161) */
        if (!last_round) {
            memset(hist, 0, (size_t)(ng + 1) * sizeof(uint32_t));
            for (uint64_t i = start; i < end; ++i) hist[group_idx[i] - base + 1]++;
            for (uint32_t g = 0; g < ng; ++g) hist[g + 1] += hist[g];
            for (uint64_t i = start; i < end; ++i) {
                uint32_t g = group_idx[i] - base;
                uint64_t dst = start + hist[g]++;
                neworder[dst] = order[i];
                out_group[dst] = g + base;
            }
        }
        start = end;
    }
    if (!last_round) memcpy(order, neworder, n * sizeof(uint32_t));
    else if (out_group) memcpy(out_group, group_idx, n * sizeof(uint32_t));
    if (ngroups) *ngroups = next_id;
    free(key); free(slot_row); free(hist); free(neworder);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* hash grouping without re-clustering, src/hashing.h:96-148, 387-422         */
/* ------------------------------------------------------------------------ */
int orc_hash_unordered(const void *bank, uint32_t bank_bytes, const uint32_t *in_group,
                       uint32_t *out_group, uint64_t n, uint32_t *ngroups)
{
    if (!valid_bytes(bank_bytes)) return -1;
    if (ngroups) *ngroups = 0;
    if (n == 0) return 0;
    uint64_t ts = 16;
    while (ts < 2 * n) ts <<= 1;
    uint32_t *slot_row = (uint32_t *)malloc(ts * sizeof(uint32_t));
    if (!slot_row) return -2;
    memset(slot_row, 0xFF, ts * sizeof(uint32_t));
    uint32_t next = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t k = ld(bank, bank_bytes, i);
        uint32_t g = in_group ? in_group[i] : 0;
        uint64_t h = mix64(k ^ ((uint64_t)g * 0x9E3779B97F4A7C15ULL)) & (ts - 1);
        for (;;) {
            uint32_t r = slot_row[h];
            if (r == 0xFFFFFFFFu) { slot_row[h] = (uint32_t)i; out_group[i] = next++; break; }
            if (ld(bank, bank_bytes, r) == k && (!in_group || in_group[r] == g)) {
                out_group[i] = out_group[r];
                break;
            }
            h = (h + 1) & (ts - 1);
        }
    }
    if (ngroups) *ngroups = next;
    free(slot_row);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* whole plans                                                               */
/* ------------------------------------------------------------------------ */
static int build_banks(const void *const *cols, const uint32_t *col_bytes, const uint32_t *bw,
                       uint32_t ncols, const uint32_t *col_order, const uint32_t *split, uint32_t nbanks,
                       uint64_t n, int hash_path, void **banks, uint32_t *bank_bytes)
{
    orc_record rec[256];
    uint32_t nrec[128];
    uint32_t order_cols[128];
    uint8_t seen[128] = {0};
    if (ncols > 128 || nbanks > 128 || ncols + nbanks > 256) return -1;
    /* col_order[k] = the column whose bits come k-th (the reference's
     * columnOrder, src/stitch_composer.cpp:568-612); NULL = 0..ncols-1 */
    for (uint32_t c = 0; c < ncols; ++c) {
        order_cols[c] = col_order ? col_order[c] : c;
        if (order_cols[c] >= ncols || seen[order_cols[c]]) return -1;
        seen[order_cols[c]] = 1;
    }
    int nr = orc_plan_records(bw, ncols, order_cols, split, nbanks, rec, nrec);
    if (nr < 0) return -1;
    uint32_t r0 = 0;
    for (uint32_t b = 0; b < nbanks; ++b) {
        orc_slice sl[256];
        for (uint32_t k = 0; k < nrec[b]; ++k) {
            const orc_record *e = &rec[r0 + k];
            sl[k].src = cols[e->final_idx];
            sl[k].src_bytes = col_bytes[e->final_idx];
            sl[k].src_bits = bw[e->final_idx];
            sl[k].start = e->start;
            sl[k].end = e->end;
        }
        bank_bytes[b] = orc_bank_bytes(split[b], hash_path);
        banks[b] = calloc(n ? n : 1, bank_bytes[b]);
        if (!banks[b]) return -2;
        int rc = orc_stitch(sl, nrec[b], banks[b], bank_bytes[b], n);
        if (rc) return rc;
        r0 += nrec[b];
    }
    return 0;
}

int orc_run_plan_sort(const void *const *cols, const uint32_t *col_bytes,
                      const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                      const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups)
{
    void *banks[128] = {0};
    uint32_t bb[128];
    if (nbanks == 0 || nbanks > 128) return -1;
    int rc = build_banks(cols, col_bytes, bw, ncols, col_order, split, nbanks, n, 0, banks, bb);
    uint32_t *g0 = NULL, *g1 = NULL;
    if (rc == 0 && n > 0) {
        g0 = (uint32_t *)malloc(n * sizeof(uint32_t));
        g1 = (uint32_t *)malloc(n * sizeof(uint32_t));
        if (!g0 || !g1) rc = -2;
    }
    if (rc == 0) {
        uint32_t *in = NULL, *out = g0;
        for (uint32_t b = 0; b < nbanks && rc == 0; ++b) {
            rc = orc_sort_round(banks[b], bb[b], order_out, in, out, NULL, n, ngroups);
            in = out;
            out = (out == g0) ? g1 : g0;
        }
        if (rc == 0 && n > 0) memcpy(group_out, in, n * sizeof(uint32_t));
    }
    free(g0); free(g1);
    for (uint32_t b = 0; b < nbanks; ++b) free(banks[b]);
    return rc;
}

int orc_run_plan_hash(const void *const *cols, const uint32_t *col_bytes,
                      const uint32_t *bw, uint32_t ncols, const uint32_t *col_order,
                      const uint32_t *split, uint32_t nbanks, uint64_t n,
                      uint32_t *order_out, uint32_t *group_out, uint32_t *ngroups)
{
    void *banks[128] = {0};
    uint32_t bb[128];
    if (nbanks == 0 || nbanks > 128) return -1;
    int rc = build_banks(cols, col_bytes, bw, ncols, col_order, split, nbanks, n, 1, banks, bb);
    uint32_t *g0 = NULL, *g1 = NULL, *idx = NULL;
    if (rc == 0 && n > 0) {
        g0 = (uint32_t *)malloc(n * sizeof(uint32_t));
        g1 = (uint32_t *)malloc(n * sizeof(uint32_t));
        idx = (uint32_t *)malloc(n * sizeof(uint32_t));
        if (!g0 || !g1 || !idx) rc = -2;
    }
    if (rc == 0) {
        uint32_t *in = NULL, *out = g0;
        for (uint32_t b = 0; b < nbanks && rc == 0; ++b) {
            int last = (b + 1 == nbanks);
            rc = orc_hash_round(banks[b], bb[b], order_out, in, last ? NULL : out, idx, n,
                                last, ngroups);
            if (!last) { in = out; out = (out == g0) ? g1 : g0; }
        }
        if (rc == 0 && n > 0) memcpy(group_out, idx, n * sizeof(uint32_t));
    }
    free(g0); free(g1); free(idx);
    for (uint32_t b = 0; b < nbanks; ++b) free(banks[b]);
    return rc;
}
