// host_api_driver.cpp -- drives the C++ host classes (include/fmcs/*.h) the way
// FastMultiColSort driver code does (build Column**, setting_t,
// compose_params_t; call SortAllColumns / HashAllColumns / run_single_plan),
// and writes the results as raw uint32 files for tests/test_host_api.py to
// compare with the oracle.
//
//   host_api_driver cpu  <outdir>                     host-only logic (no GPU)
//   host_api_driver gpu  <indir> <n> <w0> <w1> <outdir>   two columns u32/u64
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "fmcs/composer.h"
#include "fmcs/plan_enum_rrs.h"
#include "fmcs/stitch_composer.h"

using namespace multiAttrSort;

template <class T>
static std::vector<T> read_bin(const std::string &path, uint64_t n)
{
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read((char *)v.data(), n * sizeof(T));
    if (!f) {
        std::cerr << "cannot read " << path << std::endl;
        exit(2);
    }
    return v;
}

static void write_u32(const std::string &path, const std::vector<uint32_t> &v)
{
    std::ofstream f(path, std::ios::binary);
    f.write((const char *)v.data(), v.size() * sizeof(uint32_t));
}

static int cpu_mode(const std::string &out)
{
    // plan enumeration and cost model: no GPU involved
    std::vector<uint32_t> c0(8, 1), c1(8, 2);
    SpecialiedColumn<uint32_t> a;
    a.SetColumn(c0.data());
    a.SetCardinality(8192);
    SpecialiedColumn<uint64_t> b;
    b.SetColumn((uint64_t *)c1.data());
    b.SetCardinality(1ull << 33);
    Column *cols[2] = {&a, &b};
    uint32_t bw[2] = {17, 33};
    bool asc[2] = {true, true};
    compose_params_t params;
    params.bitwidth = bw;
    params.column_asc_desc = asc;
    params.colwidth_sum = 50;
    setting_t setting;
    StitchComposer sc(setting, 2, 16777216, params, cols);
    std::vector<std::vector<uint32_t>> plans1, plans2;
    sc.split_exhaustive_certain_round(50, 0, 1, 64, plans1);
    sc.split_exhaustive_certain_round(50, 0, 2, 64, plans2);
    std::vector<std::vector<uint32_t>> greedy;
    uint32_t order[2] = {0, 1};
    sc.find_greedy_plans(3, greedy, order);
    std::vector<uint32_t> best_order;
    double est = 0;
    std::vector<uint32_t> best = sc.OptimizePlan(&best_order, &est);
    std::ofstream f(out + "/cpu.txt");
    f << "plans1 " << plans1.size() << "\n";
    f << "plans2 " << plans2.size() << "\n";
    f << "greedy " << greedy.size() << "\n";
    for (auto &p : greedy) {
        uint32_t s = 0;
        for (uint32_t w : p) s += w;
        f << "greedy_sum " << s << " rounds " << p.size() << "\n";
    }
    f << "groups17 " << sc.estimateGroupNum(17, order) << "\n";
    f << "best";
    for (uint32_t w : best) f << " " << w;
    f << "\nest " << est << "\n";
    PlanEnumRRS rrs(16777216, 50, 4, {0, 1}, 2, {17, 33}, {8192, 1u << 31}, 50.0);
    rrs.Optimize();
    auto p = rrs.GetOptimalPoint();
    uint32_t s = 0;
    for (uint32_t w : p) s += w;
    f << "rrs_sum " << s << " searched " << rrs.ObtainPlans().size() << "\n";
    return 0;
}

static int gpu_mode(const std::string &in, uint64_t n, uint32_t w0, uint32_t w1, const std::string &out)
{
    std::vector<uint32_t> col0 = read_bin<uint32_t>(in + "/col0.bin", n);
    std::vector<uint64_t> col1 = read_bin<uint64_t>(in + "/col1.bin", n);
    SpecialiedColumn<uint32_t> a;
    a.SetColumn(col0.data());
    a.SetWidth(4);
    a.SetCardinality(8192);
    SpecialiedColumn<uint64_t> b;
    b.SetColumn(col1.data());
    b.SetWidth(8);
    b.SetCardinality(n);
    Column *cols[2] = {&a, &b};
    uint32_t bw[2] = {w0, w1};
    bool asc[2] = {true, true};
    compose_params_t params;
    params.bitwidth = bw;
    params.column_asc_desc = asc;
    params.colwidth_sum = w0 + w1;
    setting_t setting;

    // 1) ChainComposer on the plain columns: one round per column
    {
        ChainComposer cc(setting, 2, n, params, cols);
        cc.SortAllColumns();
        write_u32(out + "/chain_order.bin", cc.GetOrder());
        write_u32(out + "/chain_group.bin", cc.GetGroup());
    }
    // 2) StitchComposer: massaged plans through run_single_plan
    {
        StitchComposer sc(setting, 2, n, params, cols);
        uint32_t order[2] = {0, 1};
        for (auto split : std::vector<std::vector<uint32_t>>{{w0 + w1}, {6, w0 + w1 - 6}, {w0, w1}}) {
            double bd[6];
            sc.run_single_plan(order, split, bd);
            std::string tag;
            for (size_t i = 0; i < split.size(); ++i) tag += (i ? "B" : "") + std::to_string(split[i]);
            write_u32(out + "/stitch_" + tag + "_order.bin", sc.GetOrder());
            write_u32(out + "/stitch_" + tag + "_group.bin", sc.GetGroup());
            if (!(bd[3] > 0.0) || !(bd[0] > 0.0)) {
                std::cerr << "breakdown not filled" << std::endl;
                return 3;
            }
        }
        // the optimizer picks and runs a plan (SortAllColumns_Nonpack)
        sc.SortAllColumns();
        write_u32(out + "/optimized_order.bin", sc.GetOrder());
        write_u32(out + "/optimized_group.bin", sc.GetGroup());
        sc.RunAnInstance("6B44");
    }
    // 3) hash grouping: reordered (hash_type 1) and non-reordered (0)
    for (uint32_t ht : {1u, 0u}) {
        compose_params_t hp = params;
        hp.hash_type = ht;
        ChainComposer cc(setting, 2, n, hp, cols);
        cc.HashAllColumns();
        write_u32(out + "/hash" + std::to_string(ht) + "_order.bin", cc.GetOrder());
        write_u32(out + "/hash" + std::to_string(ht) + "_group.bin", cc.GetGroup());
    }
    // 4) a bank built slice by slice with the reference's two primitives
    {
        std::vector<uint64_t> bank(n, 0);
        SpecialiedColumn<uint64_t> bk;
        bk.SetColumn(bank.data());
        bk.AssembleFromColumn(&a, 1, w0, n, w0);
        bk.ShiftLeftBatch(n, w1);
        bk.AssembleFromColumn(&b, 1, w1, n, w1);
        std::vector<uint32_t> lo(n), hi(n);
        for (uint64_t i = 0; i < n; ++i) {
            lo[i] = (uint32_t)bank[i];
            hi[i] = (uint32_t)(bank[i] >> 32);
        }
        write_u32(out + "/bank_lo.bin", lo);
        write_u32(out + "/bank_hi.bin", hi);
        if (bk.GetValueAt(1) != bank[1]) return 4;
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc >= 3 && std::string(argv[1]) == "cpu") return cpu_mode(argv[2]);
    if (argc >= 7 && std::string(argv[1]) == "gpu")
        return gpu_mode(argv[2], strtoull(argv[3], nullptr, 10), (uint32_t)atoi(argv[4]), (uint32_t)atoi(argv[5]),
                        argv[6]);
    std::cerr << "usage: host_api_driver cpu <outdir> | gpu <indir> <n> <w0> <w1> <outdir>" << std::endl;
    return 1;
}
