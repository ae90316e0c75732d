// stitch_composer.cpp -- StitchComposer (include/fmcs/stitch_composer.h) and
// the GPU cost tables (include/fmcs/cost_model.h).
//
// Reference: src/stitch_composer.cpp -- constructor statistics (header
// :16-43), plan enumeration (:205-230, :1991-2125), group-number estimate
// (:1845-1867), plan costing (:2186-2378), optimizeAndRun (:3839-4013),
// RunAnInstance / TwoRoundsExhaustive (:4051-4258).  The enumeration and the
// shape of the cost function follow the reference; the cost tables are GPU
// milliseconds (GpuCostTables) instead of Haswell cycles.
#include "../../../include/fmcs/stitch_composer.h"

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace multiAttrSort {

// =============================================================== cost tables
namespace {

// Minimal reader of the flat JSON the autotuner writes: "key": number or
// "key": [numbers] or "key": [[numbers], ...].
bool json_numbers(const std::string &txt, const std::string &key, std::vector<double> &out)
{
    out.clear();
    const std::string pat = "\"" + key + "\"";
    size_t p = txt.find(pat);
    if (p == std::string::npos) return false;
    p = txt.find(':', p + pat.size());
    if (p == std::string::npos) return false;
    ++p;
    while (p < txt.size() && isspace((unsigned char)txt[p])) ++p;
    if (p >= txt.size()) return false;
    if (txt[p] != '[') {   // a scalar up to the next ',' or '}'
        const size_t e = txt.find_first_of(",}", p);
        out.push_back(strtod(txt.substr(p, e - p).c_str(), nullptr));
        return true;
    }
    size_t q = p;
    int depth = 0;
    for (; q < txt.size(); ++q) {
        if (txt[q] == '[') depth++;
        if (txt[q] == ']' && --depth == 0) break;
    }
    std::string body = txt.substr(p, q - p + 1);
    for (char &c : body)
        if (c == '[' || c == ']' || c == ',') c = ' ';
    std::istringstream is(body);
    double v;
    while (is >> v) out.push_back(v);
    return !out.empty();
}

std::string library_dir()
{
    Dl_info info;
    if (dladdr((void *)&library_dir, &info) && info.dli_fname) {
        std::string f = info.dli_fname;
        size_t s = f.rfind('/');
        if (s != std::string::npos) return f.substr(0, s);
    }
    return ".";
}

}  // namespace

bool GpuCostTables::Load(const std::string &path)
{
    std::ifstream f(path);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string txt = ss.str();
    std::vector<double> v;
    GpuCostTables t = *this;
    if (json_numbers(txt, "stitch_per_byte", v) && v.size() == 1) t.stitch_per_byte = v[0];
    if (json_numbers(txt, "gather", v) && v.size() == 3) std::copy(v.begin(), v.end(), t.gather);
    if (json_numbers(txt, "boundary", v) && v.size() == 3) std::copy(v.begin(), v.end(), t.boundary);
    if (json_numbers(txt, "msd_level", v) && v.size() == 3) std::copy(v.begin(), v.end(), t.msd_level);
    if (json_numbers(txt, "local", v) && v.size() % 3 == 0 && v.size() >= 3) {
        // rows of per-size costs (sizes 2^0 ..); missing larger sizes keep the
        // last measured per-row cost
        const int per = (int)(v.size() / 3);
        for (int b = 0; b < 3; ++b)
            for (int k = 0; k < kLocalSizes; ++k) t.local[b][k] = v[b * per + std::min(k, per - 1)];
    }
    if (json_numbers(txt, "round_fixed_ms", v) && v.size() == 1) t.round_fixed_ms = v[0];
    if (json_numbers(txt, "local_max", v) && v.size() == 1 && v[0] >= 128 && v[0] <= 8192)
        t.local_max = (uint32_t)v[0];
    *this = t;
    return true;
}

GpuCostTables GpuCostTables::Default()
{
    GpuCostTables t;
    const char *env = getenv("FMCS_TUNING");
    if (env && t.Load(env)) return t;
    t.Load(library_dir() + "/tuning/b200.json");
    return t;
}

const GpuCostTables &GpuCostTables::Cached()
{
    static const GpuCostTables tables = Default();   // read once per process
    return tables;
}

double GpuCostTables::SortGroupMs(double g, uint32_t bank_bytes, uint32_t key_bits) const
{
    if (g <= 1.0) return 0.0;
    const int b = BankIndex(bank_bytes);
    double per_mrow = 0.0;
    double rest = g;
    int levels = 0;
    const int max_levels = (int)((key_bits + 7) / 8);
    while (rest > (double)local_max && levels < max_levels) {
        rest /= 256.0;
        levels++;
        per_mrow += msd_level[b];
    }
    int k = (int)std::ceil(std::log2(std::max(1.0, std::min(rest, (double)local_max))));
    k = std::max(0, std::min(kLocalSizes - 1, k));
    per_mrow += local[b][k];
    return per_mrow * g / 1e6;
}

double GpuCostTables::SortRoundMs(uint64_t n, double g, uint32_t bank_bytes, uint32_t key_bits) const
{
    if (g < 1.0) g = 1.0;
    return ((double)n / g) * SortGroupMs(g, bank_bytes, key_bits);
}

double GpuCostTables::SortGroupMs(double g, uint32_t bank_bytes, uint32_t key_bits, const double *split,
                                  int nsplit) const
{
    if (g <= 1.0) return 0.0;
    const int b = BankIndex(bank_bytes);
    double per_mrow = 0.0;
    double rest = g;
    int levels = 0;
    const int max_levels = (int)((key_bits + 7) / 8);
    while (rest > (double)local_max && levels < max_levels) {
        levels++;
        per_mrow += msd_level[b];
        // after `levels` levels a group holds the rows of one value of its
        // top 8 * levels key bits: 256^levels parts at most, and no more than
        // those bits take distinct values
        double parts = std::pow(256.0, (double)levels);
        if (split && levels <= nsplit) parts = std::min(parts, split[levels - 1]);
        rest = g / std::max(1.0, std::min(parts, g));
    }
    int k = (int)std::ceil(std::log2(std::max(1.0, std::min(rest, (double)local_max))));
    k = std::max(0, std::min(kLocalSizes - 1, k));
    per_mrow += local[b][k];
    return per_mrow * g / 1e6;
}

double GpuCostTables::SortRoundMs(uint64_t n, double g, uint32_t bank_bytes, uint32_t key_bits, const double *split,
                                  int nsplit) const
{
    if (g < 1.0) g = 1.0;
    return ((double)n / g) * SortGroupMs(g, bank_bytes, key_bits, split, nsplit);
}

// ============================================================ StitchComposer
StitchComposer::StitchComposer(setting_t setting, uint32_t ncolumns, uint64_t nrows, compose_params_t params,
                               Column **column_values)
    : Composer(setting, ncolumns, nrows, params, column_values), tables_(GpuCostTables::Cached())
{
    // cardinality carried by each bit of each column, and the shrink factor
    // (reference: src/stitch_composer.h:16-43)
    base_col_card.resize(num_columns_);
    card_per_bit.resize(num_columns_);
    double all = 1.0;
    for (uint32_t c = 0; c < num_columns_; ++c) {
        uint64_t card = column_values_[c]->GetCardinality();
        if (card == 0) card = 1;
        base_col_card[c] = card;
        all *= (double)card;
        const uint32_t w = compose_params_.bitwidth ? compose_params_.bitwidth[c] : 8 * column_values_[c]->GetWidth();
        card_per_bit[c] = std::pow((double)card, 1.0 / (double)std::max<uint32_t>(1, w));
    }
    if (num_columns_ > 1) shrink_factor = std::pow((double)num_rows_ / all, 1.0 / (double)(num_columns_ - 1));
    if (compose_params_.colwidth_sum == 0 && compose_params_.bitwidth)
        for (uint32_t c = 0; c < num_columns_; ++c) compose_params_.colwidth_sum += compose_params_.bitwidth[c];
}

double StitchComposer::estimate_mergesort_uint16(double nitems)
{
    return GpuCostTables::Cached().SortGroupMs(nitems, 2, 16);
}
double StitchComposer::estimate_mergesort_uint32(double nitems)
{
    return GpuCostTables::Cached().SortGroupMs(nitems, 4, 32);
}
double StitchComposer::estimate_mergesort_uint64(double nitems)
{
    return GpuCostTables::Cached().SortGroupMs(nitems, 8, 64);
}

double StitchComposer::estimate_stitch(uint32_t assembleStatistics[][3], uint32_t shiftStatistics[], uint32_t nitems)
{
    // bytes moved by the fused stitch: each slice reads its source once, each
    // bank is written once
    static const double bytes[3] = {2, 4, 8};
    double moved = 0.0;
    for (int from = 0; from < 3; ++from)
        for (int to = 0; to < 3; ++to) moved += assembleStatistics[from][to] * bytes[from];
    for (int to = 0; to < 3; ++to) moved += (shiftStatistics[to] ? 1 : 0) * bytes[to];
    return GpuCostTables::Cached().stitch_per_byte * moved * (double)nitems / 1e6;
}

double StitchComposer::estimate_tuple_reconstruct(const uint32_t *bytewidths, const uint32_t column_num,
                                                  const uint64_t rows_num)
{
    const GpuCostTables &t = GpuCostTables::Cached();
    double ms = 0.0;
    for (uint32_t c = 1; c < column_num; ++c) ms += t.gather[GpuCostTables::BankIndex(bytewidths[c])] * rows_num / 1e6;
    return ms;
}

double StitchComposer::calculate_single_column_cost(const double groupsz, const uint32_t banksz_type)
{
    static const uint32_t bytes[3] = {2, 4, 8};
    return tables_.SortRoundMs(num_rows_, groupsz, bytes[std::min<uint32_t>(banksz_type, 2)],
                               8 * bytes[std::min<uint32_t>(banksz_type, 2)]);
}

double StitchComposer::estimateGroupNum(const uint32_t bit_position, const uint32_t *columnOrder)
{
    uint32_t bits = bit_position;
    double g = 1.0;
    for (uint32_t i = 0; i < num_columns_ && bits > 0; ++i) {
        const uint32_t c = columnOrder[i];
        const uint32_t w = compose_params_.bitwidth[c];
        const uint32_t take = std::min(bits, w);
        g *= std::pow(card_per_bit[c], (double)take);
        bits -= take;
    }
    return std::min(g, (double)num_rows_);
}

double StitchComposer::EstimatePlan(const uint32_t *columnOrder, const std::vector<uint32_t> &split)
{
    const uint32_t *bw = compose_params_.bitwidth;
    double ms = 0.0;
    uint32_t prefix = 0;
    // which columns feed each bank (for the stitch bytes)
    std::vector<uint32_t> colstart(num_columns_ + 1, 0);
    for (uint32_t i = 0; i < num_columns_; ++i) colstart[i + 1] = colstart[i] + bw[columnOrder[i]];
    for (size_t r = 0; r < split.size(); ++r) {
        const uint32_t w = split[r];
        const uint32_t B = w <= 16 ? 2 : (w <= 32 ? 4 : 8);
        const int bi = GpuCostTables::BankIndex(B);
        double src_bytes = 0.0;
        for (uint32_t i = 0; i < num_columns_; ++i)
            if (colstart[i] < prefix + w && colstart[i + 1] > prefix) src_bytes += column_values_[columnOrder[i]]->GetWidth();
        ms += tables_.stitch_per_byte * (src_bytes + B) * num_rows_ / 1e6;
        if (r > 0) ms += tables_.gather[bi] * num_rows_ / 1e6;
        const double groups = r == 0 ? 1.0 : estimateGroupNum(prefix, columnOrder);
        // distinct values of the bank's top 8, 16, ... bits inside a group:
        // how far each radix level can split it (the reference's per-bit
        // cardinality model, src/stitch_composer.h:16-43)
        double split_parts[8];
        const int nsplit = (int)std::min<uint32_t>(8, (w + 7) / 8);
        for (int l = 0; l < nsplit; ++l)
            split_parts[l] = estimateGroupNum(prefix + std::min<uint32_t>(w, 8u * (uint32_t)(l + 1)), columnOrder) /
                             groups;
        ms += tables_.SortRoundMs(num_rows_, (double)num_rows_ / groups, B, w, split_parts, nsplit);
        ms += tables_.boundary[bi] * num_rows_ / 1e6;
        ms += tables_.round_fixed_ms;
        prefix += w;
    }
    return ms;
}

void StitchComposer::split_exhaustive_certain_round(int n, int curRound, const int round_num, const int maxValue,
                                                    std::vector<std::vector<uint32_t>> &split_enum)
{
    if (curRound == round_num - 1) {
        if (n <= 0 || n > maxValue) return;
        partitions_[curRound] = (uint32_t)n;
        split_enum.emplace_back(partitions_, partitions_ + round_num);
        return;
    }
    for (int i = std::min(n, maxValue); i > 0; --i) {
        partitions_[curRound] = (uint32_t)i;
        if (n - i > 0) split_exhaustive_certain_round(n - i, curRound + 1, round_num, maxValue, split_enum);
    }
}

void StitchComposer::find_greedy_plans(uint32_t round_num, std::vector<std::vector<uint32_t>> &validPlans,
                                       const uint32_t *columnOrder)
{
    // enumerate bank-size categories (16/32/64 per round) and, round by
    // round, cut where the NEXT round's sort is cheapest
    const uint32_t total = compose_params_.colwidth_sum;
    static const uint32_t lo_bits[3] = {1, 17, 33}, hi_bits[3] = {16, 32, 64};
    std::vector<uint32_t> cate(round_num, 0);
    for (;;) {
        std::vector<uint32_t> plan;
        uint32_t offset = 0;
        bool ok = true;
        for (uint32_t r = 0; r + 1 < round_num && ok; ++r) {
            const uint32_t mn = offset + lo_bits[cate[r]], mx = std::min(total - 1, offset + hi_bits[cate[r]]);
            if (mn > mx) {
                ok = false;
                break;
            }
            const uint32_t nb = hi_bits[cate[r + 1]] == 16 ? 2 : (hi_bits[cate[r + 1]] == 32 ? 4 : 8);
            double best = std::numeric_limits<double>::max();
            uint32_t best_pos = mn;
            for (uint32_t pos = mn; pos <= mx; ++pos) {
                const double g = (double)num_rows_ / estimateGroupNum(pos, columnOrder);
                const double c = tables_.SortRoundMs(num_rows_, g, nb, 8 * nb);
                if (c <= best) {
                    best = c;
                    best_pos = pos;
                }
            }
            plan.push_back(best_pos - offset);
            offset = best_pos;
        }
        if (ok && offset < total) {
            const uint32_t last = total - offset;
            const uint32_t c = cate[round_num - 1];
            if (last >= lo_bits[c] && last <= hi_bits[c]) {
                plan.push_back(last);
                validPlans.push_back(plan);
            }
        }
        // next category vector (base-3 counter)
        uint32_t i = 0;
        while (i < round_num && ++cate[i] == 3) cate[i++] = 0;
        if (i == round_num) break;
    }
}

void StitchComposer::permutations(std::vector<uint32_t> &arr, uint32_t k, std::vector<std::vector<uint32_t>> &out)
{
    if (k + 1 >= arr.size()) {
        out.push_back(arr);
        return;
    }
    for (uint32_t i = k; i < arr.size(); ++i) {
        std::swap(arr[k], arr[i]);
        permutations(arr, k + 1, out);
        std::swap(arr[k], arr[i]);
    }
}

std::vector<uint32_t> StitchComposer::OptimizePlan(std::vector<uint32_t> *columnOrder, double *est_ms)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<uint32_t> base(num_columns_);
    for (uint32_t i = 0; i < num_columns_; ++i) base[i] = i;
    std::vector<std::vector<uint32_t>> orders;
    if (compose_params_.ordered == 0)
        permutations(base, 0, orders);   // GROUP BY: any column order
    else
        orders.push_back(base);
    const uint32_t total = compose_params_.colwidth_sum;
    const uint32_t max_rounds = (uint32_t)std::ceil((2.0 * total - 2.0) / 16.0);
    double best = std::numeric_limits<double>::max();
    std::vector<uint32_t> best_plan, best_order;
    for (const auto &ord : orders) {
        for (uint32_t rounds = 1; rounds <= std::max<uint32_t>(1, max_rounds); ++rounds) {
            std::vector<std::vector<uint32_t>> plans;
            if (rounds <= 2)
                split_exhaustive_certain_round((int)total, 0, (int)rounds, 64, plans);
            else
                find_greedy_plans(rounds, plans, ord.data());
            for (const auto &p : plans) {
                const double c = EstimatePlan(ord.data(), p);
                if (c < best) {
                    best = c;
                    best_plan = p;
                    best_order = ord;
                }
            }
            // early stop: optimization time above 1% of the best plan's cost
            // (THRESHOLD_PERC, src/params.h:90; src/stitch_composer.cpp:3945-3953)
            const double spent = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (!best_plan.empty() && rounds >= 2 && spent > 0.01 * best) break;
        }
    }
    setting_.time_optimization =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (columnOrder) *columnOrder = best_order;
    if (est_ms) *est_ms = best;
    return best_plan;
}

double StitchComposer::run_plan(const uint32_t *columnOrder, const std::vector<uint32_t> &split, bool hash,
                                double *breakdown)
{
    ensure_buffers();
    fmcs_ctx *ctx = GetContext();
    std::vector<const void *> cols(num_columns_);
    std::vector<uint32_t> cb(num_columns_);
    for (uint32_t c = 0; c < num_columns_; ++c) {
        cols[c] = column_values_[c]->GetColumn();
        cb[c] = column_values_[c]->GetWidth();
    }
    if (breakdown) fmcs_profile(ctx, 1);
    const auto t0 = std::chrono::steady_clock::now();
    uint32_t ng = 0;
    detail::check(fmcs_run_plan(ctx, cols.data(), cb.data(), compose_params_.bitwidth, num_columns_, columnOrder,
                                split.data(), (uint32_t)split.size(), num_rows_, hash ? 1 : 0, d_order_, d_group_[0],
                                &ng),
                  "run_single_plan");
    const double total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    final_group_ = 0;
    ngroups_ = ng;
    group_info_.ngroups = ng;
    group_info_.sum_group_size = (uint32_t)num_rows_;
    if (breakdown) {
        for (int i = 0; i < 6; ++i) breakdown[i] = 0.0;
        char buf[1 << 14];
        if (fmcs_profile_report(ctx, buf, sizeof(buf)) == FMCS_OK) {
            // {"name": {"launches": n, "ms": t, "units": u}, ..., "_round_ms": [r0, r1, ...]}
            std::string s(buf);
            size_t p = 0;
            while ((p = s.find('"', p)) != std::string::npos) {
                size_t q = s.find('"', p + 1);
                const std::string name = s.substr(p + 1, q - p - 1);
                if (name == "_round_ms") {
                    std::vector<double> r;
                    if (json_numbers(s, "_round_ms", r) && !r.empty()) breakdown[4] = r[0];
                    break;
                }
                size_t m = s.find("\"ms\":", q);
                const double ms = strtod(s.c_str() + m + 5, nullptr);
                if (name == "stitch") breakdown[0] += ms;
                else if (name == "gather") breakdown[1] += ms;
                else if (name == "boundary_scan") { breakdown[2] += ms; breakdown[5] += ms; }
                else breakdown[3] += ms;
                p = s.find('}', m) + 1;
            }
        }
        fmcs_profile(ctx, 0);
        setting_.time_stitching = breakdown[0];
        setting_.time_multipass_sort = breakdown[3];
        setting_.time_orderGroupInfo = breakdown[2];
    }
    return total;
}

double StitchComposer::run_single_plan(uint32_t *columnOrder, std::vector<uint32_t> &curSplit, double *breakdown)
{
    return run_plan(columnOrder, curSplit, false, breakdown);
}

double StitchComposer::run_single_plan_hash(uint32_t *columnOrder, std::vector<uint32_t> &curSplit,
                                            double *breakdown)
{
    return run_plan(columnOrder, curSplit, true, breakdown);
}

std::vector<uint32_t> StitchComposer::parse_plan(const std::string &instance)
{
    // "50" -> {50}; "6B44" -> {6, 44} (src/stitch_composer.cpp:4098-4110)
    std::vector<uint32_t> out;
    std::string tok;
    for (char c : instance + "B") {
        if (c == 'B' || c == 'b') {
            if (!tok.empty()) out.push_back((uint32_t)std::stoul(tok));
            tok.clear();
        } else {
            tok += c;
        }
    }
    return out;
}

void StitchComposer::SortAllColumns_Nonpack()
{
    const auto t0 = std::chrono::steady_clock::now();
    multiRoundSorting();
    const double base_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "[INFO ] The baseline plan is [";
    for (uint32_t i = 0; i < num_columns_; ++i) std::cout << compose_params_.bitwidth[i] << ", ";
    std::cout << "]\n[INFO ] Baseline output <optimization time, other time, [massaging time, execution time]> in ms:\n"
              << 0.0 << ", " << base_ms << ", [0.0, " << base_ms << "]\n";
    optimizeAndRun();
}

void StitchComposer::optimizeAndRun()
{
    std::vector<uint32_t> order;
    double est = 0.0;
    std::vector<uint32_t> plan = OptimizePlan(&order, &est);
    double breakdown[6];
    const double total = run_plan(order.data(), plan, false, breakdown);
    std::cout << "[INFO ] The optimized plan is [";
    for (uint32_t b : plan) std::cout << b << ", ";
    std::cout << "] under the ordering <";
    for (uint32_t c : order) std::cout << c << ", ";
    std::cout << ">\n[INFO ] Breakdown <optimization time, other time, [massaging time, execution time]> in ms:\n"
              << setting_.time_optimization << ", " << total << ", [" << breakdown[0] << ", " << (total - breakdown[0])
              << "]\n";
}

void StitchComposer::RunAnInstance(std::string instance)
{
    uint32_t order[2] = {0, 1};
    const uint32_t w0 = compose_params_.bitwidth[0], w1 = compose_params_.bitwidth[1];
    std::vector<uint32_t> warm{w0 + w1};
    for (int i = 0; i < 5; ++i) run_plan(order, warm, false, nullptr);   // warm-up, as the reference
    const double mrows = (double)num_rows_ / 1e6;
    double bb[6];
    std::vector<uint32_t> base{w0, w1};
    run_single_plan(order, base, bb);
    std::cout << "0, 0, " << bb[4] / mrows << ", " << (bb[3] - bb[4]) / mrows << ", " << bb[1] / mrows << ", "
              << bb[2] / mrows << std::endl;
    std::vector<uint32_t> plan = parse_plan(instance);
    double bp[6];
    run_single_plan(order, plan, bp);
    std::cout << "1, " << bp[0] / mrows << ", " << bp[4] / mrows << ", " << (bp[3] - bp[4]) / mrows << ", "
              << bp[1] / mrows << ", " << bp[2] / mrows << std::endl;
}

void StitchComposer::TwoRoundsExhaustive()
{
    uint32_t order[2] = {0, 1};
    const int w0 = (int)compose_params_.bitwidth[0], w1 = (int)compose_params_.bitwidth[1];
    std::vector<uint32_t> warm{(uint32_t)(w0 + w1)};
    for (int i = 0; i < 5; ++i) run_plan(order, warm, false, nullptr);
    const double mrows = (double)num_rows_ / 1e6;
    for (int s = -w1; s <= w0; ++s) {
        std::vector<uint32_t> split;
        if (w0 - s > 0) split.push_back((uint32_t)(w0 - s));
        if (w1 + s > 0) split.push_back((uint32_t)(w1 + s));
        double b[6];
        const double total = run_single_plan(order, split, b);
        std::cout << s << ", " << b[4] / mrows << ", " << (b[3] - b[4]) / mrows << ", " << (total - b[3]) / mrows
                  << std::endl;
    }
}

void StitchComposer::ExhaustiveSearch()
{
    std::vector<uint32_t> order(num_columns_);
    for (uint32_t i = 0; i < num_columns_; ++i) order[i] = i;
    const uint32_t total = compose_params_.colwidth_sum;
    double best = std::numeric_limits<double>::max();
    std::vector<uint32_t> best_plan;
    for (int rounds = 1; rounds <= 2; ++rounds) {
        std::vector<std::vector<uint32_t>> plans;
        split_exhaustive_certain_round((int)total, 0, rounds, 64, plans);
        for (auto &p : plans) {
            const double ms = run_plan(order.data(), p, false, nullptr);
            if (ms < best) {
                best = ms;
                best_plan = p;
            }
        }
    }
    std::cout << "[INFO ] Exhaustive best plan [";
    for (uint32_t b : best_plan) std::cout << b << ", ";
    std::cout << "] in " << best << " ms" << std::endl;
}

void StitchComposer::CostModelComparison()
{
    std::vector<uint32_t> order(num_columns_);
    for (uint32_t i = 0; i < num_columns_; ++i) order[i] = i;
    const uint32_t total = compose_params_.colwidth_sum;
    for (int rounds = 1; rounds <= 2; ++rounds) {
        std::vector<std::vector<uint32_t>> plans;
        split_exhaustive_certain_round((int)total, 0, rounds, 64, plans);
        for (auto &p : plans) {
            const double est = EstimatePlan(order.data(), p);
            const double act = run_plan(order.data(), p, false, nullptr);
            for (size_t i = 0; i < p.size(); ++i) std::cout << (i ? "B" : "") << p[i];
            std::cout << ", " << est << ", " << act << std::endl;
        }
    }
}

void StitchComposer::HashAllColumns()
{
    std::vector<uint32_t> order;
    std::vector<uint32_t> plan = OptimizePlan(&order, nullptr);
    run_plan(order.data(), plan, true, nullptr);
}

void StitchComposer::RunAnInstance_hash(std::string instance)
{
    uint32_t order[2] = {0, 1};
    const uint32_t w0 = compose_params_.bitwidth[0], w1 = compose_params_.bitwidth[1];
    const double mrows = (double)num_rows_ / 1e6;
    std::vector<uint32_t> base{w0, w1};
    double bb[6];
    const double tb = run_single_plan_hash(order, base, bb);
    std::cout << "Summary of baseline <total, massage, first round hash, other round hash>\n"
              << (tb - bb[0]) / mrows << ", 0, " << bb[4] / mrows << ", " << (bb[3] - bb[4]) / mrows << std::endl;
    std::vector<uint32_t> plan = parse_plan(instance);
    double bp[6];
    const double tp = run_single_plan_hash(order, plan, bp);
    std::cout << "Summary of specific instance <total, massage, first round hash, other round hash>\n"
              << tp / mrows << ", " << bp[0] / mrows << ", " << bp[4] / mrows << ", " << (bp[3] - bp[4]) / mrows
              << std::endl;
}

void StitchComposer::TwoRoundsExhaustive_hash()
{
    uint32_t order[2] = {0, 1};
    const int w0 = (int)compose_params_.bitwidth[0], w1 = (int)compose_params_.bitwidth[1];
    const double mrows = (double)num_rows_ / 1e6;
    for (int s = -w1; s <= w0; ++s) {
        std::vector<uint32_t> split;
        if (w0 - s > 0) split.push_back((uint32_t)(w0 - s));
        if (w1 + s > 0) split.push_back((uint32_t)(w1 + s));
        double b[6];
        const double total = run_single_plan_hash(order, split, b);
        std::cout << s << ", " << total / mrows << ", " << b[0] / mrows << ", " << b[3] / mrows << std::endl;
    }
}

}  // namespace multiAttrSort

// ================================================================ C ABI
namespace {

// A composer over statistics only (bit widths, cardinalities, storage widths):
// no column data is touched.
struct StatComposer {
    std::vector<multiAttrSort::SpecialiedColumn<uint64_t>> cols;
    std::vector<multiAttrSort::Column *> ptrs;
    std::vector<uint32_t> widths;
    multiAttrSort::compose_params_t params;
    multiAttrSort::setting_t setting;
    std::unique_ptr<multiAttrSort::StitchComposer> sc;

    bool init(const uint32_t *bw, const uint64_t *cardinality, const uint32_t *col_bytes, uint32_t ncols, uint64_t n,
              int ordered)
    {
        cols.resize(ncols);
        ptrs.resize(ncols);
        widths.assign(bw, bw + ncols);
        uint32_t sum = 0;
        for (uint32_t c = 0; c < ncols; ++c) {
            if (bw[c] == 0 || bw[c] > 64) return false;
            cols[c].SetWidth(col_bytes[c]);
            cols[c].SetCardinality(cardinality[c]);
            ptrs[c] = &cols[c];
            sum += bw[c];
        }
        params.bitwidth = widths.data();
        params.colwidth_sum = sum;
        params.ordered = ordered ? 1 : 0;
        sc.reset(new multiAttrSort::StitchComposer(setting, ncols, n, params, ptrs.data()));
        return true;
    }
};

}  // namespace

extern "C" FMCS_API int fmcs_estimate_plan(const uint32_t *bw, const uint64_t *cardinality, const uint32_t *col_bytes,
                                           uint32_t ncols, uint64_t n, const uint32_t *col_order,
                                           const uint32_t *split, uint32_t nbanks, double *est_ms)
{
    if (!bw || !cardinality || !col_bytes || !split || !est_ms || ncols == 0 || ncols > 64 || nbanks == 0)
        return FMCS_E_INVAL;
    try {
        std::vector<uint32_t> order(ncols);
        std::vector<bool> seen(ncols, false);
        for (uint32_t c = 0; c < ncols; ++c) {
            order[c] = col_order ? col_order[c] : c;
            if (order[c] >= ncols || seen[order[c]]) return FMCS_E_INVAL;
            seen[order[c]] = true;
        }
        uint64_t total = 0, sum = 0;
        for (uint32_t c = 0; c < ncols; ++c) total += bw[c];
        for (uint32_t b = 0; b < nbanks; ++b) {
            if (split[b] == 0 || split[b] > 64) return FMCS_E_INVAL;
            sum += split[b];
        }
        if (sum != total) return FMCS_E_INVAL;
        StatComposer st;
        if (!st.init(bw, cardinality, col_bytes, ncols, n, 1)) return FMCS_E_INVAL;
        *est_ms = st.sc->EstimatePlan(order.data(), std::vector<uint32_t>(split, split + nbanks));
        return FMCS_OK;
    } catch (...) {
        return FMCS_E_INVAL;
    }
}

extern "C" FMCS_API int fmcs_optimize_plan(const uint32_t *bw, const uint64_t *cardinality, const uint32_t *col_bytes,
                                           uint32_t ncols, uint64_t n, int ordered, uint32_t *split_out,
                                           uint32_t max_banks, uint32_t *nbanks_out, uint32_t *col_order_out,
                                           double *est_ms)
{
    using namespace multiAttrSort;
    if (!bw || !cardinality || !col_bytes || !split_out || !nbanks_out || ncols == 0 || ncols > 64)
        return FMCS_E_INVAL;
    try {
        StatComposer st;
        if (!st.init(bw, cardinality, col_bytes, ncols, n, ordered)) return FMCS_E_INVAL;
        std::vector<uint32_t> order;
        double est = 0.0;
        std::vector<uint32_t> plan = st.sc->OptimizePlan(&order, &est);
        if (plan.empty() || plan.size() > max_banks) return FMCS_E_INVAL;
        for (size_t i = 0; i < plan.size(); ++i) split_out[i] = plan[i];
        *nbanks_out = (uint32_t)plan.size();
        if (col_order_out)
            for (uint32_t c = 0; c < ncols; ++c) col_order_out[c] = order[c];
        if (est_ms) *est_ms = est;
        return FMCS_OK;
    } catch (...) {
        return FMCS_E_INVAL;
    }
}
