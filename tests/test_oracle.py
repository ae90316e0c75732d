"""The oracle (CPU restatement) against the reference: the committed golden
fixtures produced by the reference's own composer, the reference's 9-tuple
known-answer case, and -- where the reference harness is built -- live
comparisons on seeded inputs."""
import numpy as np
import pytest

from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O
from tests.golden_util import case_id, digest, load_cases

CASES = load_cases()


@pytest.mark.parametrize("c", CASES, ids=[case_id(c) for c in CASES])
def test_oracle_matches_golden(c):
    run = O.run_plan_sort if c["path"] == "sort" else O.run_plan_hash
    order, group, ng = run(c["cols"], c["bw"], c["split"])
    assert digest(order) == c["order_sha256"]
    assert digest(group) == c["group_sha256"]
    assert ng == c["ngroups"]
    if c["order"] is not None:
        assert np.array_equal(order, c["order"])
        assert np.array_equal(group, c["group"])


def test_subgroup_known_answer():
    # tests/subgroup_test.cpp:98-145: hash grouping of two columns equals the
    # grouping of their stitched value; first-appearance ids
    c1 = np.array([100, 200, 200, 200, 100, 100, 300, 100, 100], np.uint32)
    c2 = np.array([1000, 2000, 2000, 1000, 2000, 1000, 3000, 4000, 4000], np.uint32)
    o1, g1, n1 = O.run_plan_hash([c1, c2], [32, 32], [64])
    assert list(g1) == [0, 1, 1, 2, 3, 0, 4, 5, 5] and n1 == 6
    o2, g2, n2 = O.run_plan_hash([c1, c2], [32, 32], [32, 32])
    assert n2 == 6
    # same partition of rows into groups either way
    part1 = sorted(tuple(sorted(np.nonzero(g1 == g)[0])) for g in range(n1))
    part2 = sorted(tuple(sorted(o2[np.nonzero(g2 == g)[0]])) for g in range(n2))
    assert part1 == part2


def test_plan_records():
    assert O.plan_records([17, 33], [50]) == [[(0, 1, 17), (1, 1, 33)]]
    assert O.plan_records([17, 33], [6, 44]) == [[(0, 1, 6)], [(0, 7, 17), (1, 1, 33)]]
    assert O.plan_records([17, 33], [20, 30]) == [[(0, 1, 17), (1, 1, 3)], [(1, 4, 33)]]
    with pytest.raises(ValueError):
        O.plan_records([17, 33], [40])
    assert O.bank_bytes(8) == 2 and O.bank_bytes(8, hash_path=True) == 1
    assert O.bank_bytes(17) == 4 and O.bank_bytes(33) == 8


def test_sort_round_properties():
    rng = np.random.default_rng(5)
    bank = rng.integers(0, 1 << 12, size=5000, dtype=np.uint64).astype(np.uint16)
    order, group, keys, ng = O.sort_round(bank)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert np.array_equal(bank[order], keys)
    # stable: equal keys keep ascending oid
    same = keys[1:] == keys[:-1]
    assert np.all(order[1:][same] > order[:-1][same])
    assert ng == len(np.unique(bank))


need_ref = pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")


@need_ref
@pytest.mark.parametrize("src_bytes,bank_bytes", [(2, 2), (2, 4), (4, 4), (4, 8), (8, 8), (2, 8), (8, 4),
                                                  (1, 2), (4, 2)])
def test_stitch_vs_reference(src_bytes, bank_bytes):
    rng = np.random.default_rng(src_bytes * 10 + bank_bytes)
    n = 1003
    bits = min(8 * src_bytes, 40)
    src = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.dtype(f"u{src_bytes}"))
    other = rng.integers(0, 1 << 7, size=n, dtype=np.uint64).astype(np.dtype(f"u{src_bytes}"))
    cap = 8 * bank_bytes
    for start, end in ((1, min(bits, cap - 7)), (3, min(bits, 9)), (bits - 2, bits)):
        if end < start:
            continue
        sl = [(other, 7, 2, 6), (src, bits, start, end)]
        if 5 + end - start + 1 > cap:
            sl = sl[1:]
        mine = O.stitch(sl, bank_bytes, n)
        ref = O.ref_stitch(sl, bank_bytes, n)
        assert np.array_equal(mine, ref)


@need_ref
@pytest.mark.parametrize("split", [[17, 33], [50], [3, 47], [12, 38], [16, 34]])
def test_sort_plan_vs_reference_live(split):
    cols, bw = W.cols_17b33(1 << 16, seed_index=7)
    o, g, ng = O.run_plan_sort(cols, bw, split)
    ro, rg, _ = O.ref_run_plan_sort(cols, bw, split)
    assert np.array_equal(g, rg)
    assert np.array_equal(o, O.canonicalize(ro, rg))


@need_ref
def test_sort_round_vs_reference_live():
    rng = np.random.default_rng(11)
    n = 40000
    b0 = rng.integers(0, 300, size=n, dtype=np.uint64).astype(np.uint16)
    b1 = rng.integers(0, 1 << 30, size=n, dtype=np.uint64).astype(np.uint32)
    o0, g0, _, _ = O.sort_round(b0)
    ro0, rg0 = O.ref_sort_round(b0, 9)
    assert np.array_equal(g0, rg0)
    assert np.array_equal(o0, O.canonicalize(ro0, rg0))
    o1, g1, _, _ = O.sort_round(b1, order=o0, in_group=g0)
    ro1, rg1 = O.ref_sort_round(b1, 30, order=o0, in_group=g0)
    assert np.array_equal(g1, rg1)
    assert np.array_equal(o1, O.canonicalize(ro1, rg1))


@need_ref
@pytest.mark.parametrize("split", [[8, 12, 7], [27], [8, 19]])
def test_hash_plan_vs_reference_live(split):
    cols, bw = W.cols_uniform(32768, [8, 12, 7], seed_index=12, distinct=[16, 300, 0])
    o, g, ng = O.run_plan_hash(cols, bw, split)
    ro, rg, _ = O.ref_run_plan_hash(cols, bw, split)
    assert np.array_equal(o, ro) and np.array_equal(g, rg)


@need_ref
@pytest.mark.parametrize("path", ["sort", "hash"])
@pytest.mark.parametrize("col_order,split", [([2, 0, 1], [27]), ([1, 2, 0], [19, 8]), ([0, 2, 1], [8, 19])])
def test_plan_column_order_vs_reference_live(path, col_order, split):
    """A GROUP BY column order (src/stitch_composer.cpp:15-35, 3877-3882): the
    oracle's col_order against the reference run on the columns permuted the
    same way (its records take final_idx = columnOrder[k],
    src/stitch_composer.cpp:568-612)."""
    cols, bw = W.cols_uniform(32768, [8, 12, 7], seed_index=13, distinct=[16, 300, 0])
    pc = [cols[c] for c in col_order]
    pb = [bw[c] for c in col_order]
    if path == "sort":
        o, g, ng = O.run_plan_sort(cols, bw, split, col_order=col_order)
        ro, rg, _ = O.ref_run_plan_sort(pc, pb, split)
        assert np.array_equal(g, rg) and np.array_equal(o, O.canonicalize(ro, rg))
    else:
        o, g, ng = O.run_plan_hash(cols, bw, split, col_order=col_order)
        ro, rg, _ = O.ref_run_plan_hash(pc, pb, split)
        assert np.array_equal(o, ro) and np.array_equal(g, rg)
    assert ng == int(g.max()) + 1


def test_plan_column_order_rejects_bad_orders():
    cols, bw = W.cols_uniform(100, [8, 12, 7], seed_index=13)
    for bad in ([0, 0, 1], [0, 1, 3]):
        with pytest.raises(RuntimeError):
            O.run_plan_sort(cols, bw, [27], col_order=bad)
