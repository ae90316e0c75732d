"""The C++ host classes (include/fmcs/: Column, ChainComposer, StitchComposer,
PlanEnumRRS), driven like FastMultiColSort's own driver code by
tests/cpp/host_api_driver.cpp, against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("drv") / "host_api_driver"
    lib_dir = os.path.dirname(capi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_api_driver.cpp"), "-L" + lib_dir, "-lfmcs",
                    "-Wl,-rpath," + lib_dir, "-o", str(out)], check=True)
    return str(out)


def test_host_logic_without_gpu(driver, tmp_path):
    subprocess.run([driver, "cpu", str(tmp_path)], check=True)
    kv = {}
    for line in open(tmp_path / "cpu.txt"):
        parts = line.split()
        kv.setdefault(parts[0], []).append(parts[1:])
    assert kv["plans1"][0] == ["1"]           # [50]
    assert kv["plans2"][0] == ["49"]          # [k, 50-k], k = 1..49
    assert int(kv["greedy"][0][0]) >= 1
    for g in kv["greedy_sum"]:
        assert g[0] == "50" and g[2] == "3"
    assert float(kv["groups17"][0][0]) == pytest.approx(8192, rel=1e-6)
    best = [int(x) for x in kv["best"][0]]
    assert sum(best) == 50 and all(1 <= w <= 64 for w in best)
    assert kv["rrs_sum"][0][0] == "50"


@pytest.mark.gpu
def test_host_classes_on_gpu(driver, tmp_path):
    n = 200_003
    cols, bw = W.cols_17b33(n, seed_index=41)
    cols[0].tofile(tmp_path / "col0.bin")
    cols[1].tofile(tmp_path / "col1.bin")
    subprocess.run([driver, "gpu", str(tmp_path), str(n), "17", "33", str(tmp_path)], check=True)

    def rd(name):
        return np.fromfile(tmp_path / name, dtype=np.uint32)

    o, g, _ = O.run_plan_sort(cols, bw, [17, 33])
    assert np.array_equal(rd("chain_order.bin"), o) and np.array_equal(rd("chain_group.bin"), g)
    for split in ([50], [6, 44], [17, 33]):
        tag = "B".join(map(str, split))
        o, g, _ = O.run_plan_sort(cols, bw, split)
        assert np.array_equal(rd(f"stitch_{tag}_order.bin"), o), tag
        assert np.array_equal(rd(f"stitch_{tag}_group.bin"), g), tag
    # whatever plan the optimizer picked, the sorted result is the same
    o, g, _ = O.run_plan_sort(cols, bw, [50])
    assert np.array_equal(rd("optimized_order.bin"), o)
    assert np.array_equal(rd("optimized_group.bin"), g)
    # hash grouping, reordered: the oracle's two-round plan
    o, g, _ = O.run_plan_hash(cols, bw, [17, 33])
    assert np.array_equal(rd("hash1_order.bin"), o) and np.array_equal(rd("hash1_group.bin"), g)
    # non-reordered: first appearance of the (col0, col1) pair in row order
    g0, _ = O.hash_unordered(cols[0])
    g1, _ = O.hash_unordered(cols[1], g0)
    assert np.array_equal(rd("hash0_group.bin"), g1)
    assert np.array_equal(rd("hash0_order.bin"), np.arange(n, dtype=np.uint32))
    # slice-at-a-time bank = the fused stitch
    bank = O.stitch([(cols[0], 17, 1, 17), (cols[1], 33, 1, 33)], 8, n)
    got = rd("bank_lo.bin").astype(np.uint64) | (rd("bank_hi.bin").astype(np.uint64) << np.uint64(32))
    assert np.array_equal(got, bank)
