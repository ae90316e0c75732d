"""Parity at the workloads' own sizes, through the C ABI:

* 17B33, 16,777,216 rows, plans [50] and [17,33]: against the reference's own
  composer (the reference harness, ties canonicalised to ascending oid);
* the Zipf-segmented shape, 67,108,864 rows (20-bit Zipf(1.0) codes, 24-bit
  and 40-bit uniform): the per-column plan [20,24,40] and the cost model's
  massaged plan against the oracle;
* the wide table, 60,000,000 rows of 2/1/12/12/32/7-bit columns: the cost
  model's ORDER BY plan against the oracle, and its GROUP BY plan (a
  non-identity column order through the hash rounds) against the oracle's
  hash plan with the same column order;
* the many-instances shape (4,096 instances, about 640M rows, one
  fmcs_run_batch call): twenty instances across the size range against the
  oracle, and the whole batch against the same plan run per instance.

The reference is unstable among equal keys (src/composer.cpp:490-589); its
order is compared after sorting the oids of each final group ascending, which
is the order the stable GPU sort gives (src/composer.cpp:1222-1408 for the
rounds, src/hashing.h:289-385 for the hash rounds)."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

N_17B33 = 16_777_216
N_ZIPF = 67_108_864
WIDE_BITS = [2, 1, 12, 12, 32, 7]
WIDE_DISTINCT = [3, 2, 2526, 2526, 0, 100]   # 0: uniform 32-bit codes
N_WIDE = 60_000_000


@pytest.fixture(scope="module")
def data_17b33():
    return W.cols_17b33(N_17B33)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("split", [[50], [17, 33]])
def test_17b33_full_size_vs_reference(ctx, data_17b33, split):
    cols, bw = data_17b33
    order = np.zeros(N_17B33, np.uint32)
    group = np.zeros(N_17B33, np.uint32)
    ng = ctx.run_plan(cols, bw, split, order, group)
    r_order, r_group, _ = O.ref_run_plan_sort(cols, bw, split, final_groups=True)
    assert np.array_equal(group, r_group)
    assert ng == int(r_group[-1]) + 1
    assert np.array_equal(order, O.canonicalize(r_order, r_group))


@pytest.fixture(scope="module")
def data_zipf():
    cols, bw = W.cols_zipf(N_ZIPF)
    o, g, ng = O.run_plan_sort(cols, bw, bw)
    return cols, bw, (o, g, ng)


def zipf_plans(cols, bw):
    sizes = np.bincount(cols[0].astype(np.int64), minlength=1 << 20)
    card = [capi.effective_cardinality(sizes), 1 << 24, N_ZIPF]
    plan, corder, _ = capi.optimize_plan(bw, card, [4, 4, 8], N_ZIPF)
    assert corder == [0, 1, 2]
    return [list(bw), plan]


def test_zipf_64m_plans_vs_oracle(ctx, data_zipf):
    cols, bw, (o_ref, g_ref, ng_ref) = data_zipf
    for split in zipf_plans(cols, bw):
        order = np.zeros(N_ZIPF, np.uint32)
        group = np.zeros(N_ZIPF, np.uint32)
        ng = ctx.run_plan(cols, bw, split, order, group)
        assert ng == ng_ref, split
        assert np.array_equal(order, o_ref), split
        assert np.array_equal(group, g_ref), split


@pytest.fixture(scope="module")
def data_wide():
    cols, bw = W.cols_uniform(N_WIDE, WIDE_BITS, seed_index=4, distinct=WIDE_DISTINCT)
    card = [k if k else N_WIDE for k in WIDE_DISTINCT]
    cb = [c.dtype.itemsize for c in cols]
    osplit, _, _ = capi.optimize_plan(bw, card, cb, N_WIDE, ordered=True)
    gsplit, gorder, _ = capi.optimize_plan(bw, card, cb, N_WIDE, ordered=False)
    return cols, bw, osplit, gsplit, gorder


def test_wide_60m_order_by_vs_oracle(ctx, data_wide):
    cols, bw, osplit, _, _ = data_wide
    order = np.zeros(N_WIDE, np.uint32)
    group = np.zeros(N_WIDE, np.uint32)
    ng = ctx.run_plan(cols, bw, osplit, order, group)
    o, g, n_ref = O.run_plan_sort(cols, bw, osplit)
    assert ng == n_ref
    assert np.array_equal(order, o)
    assert np.array_equal(group, g)


def test_wide_60m_group_by_hash_vs_oracle(ctx, data_wide):
    cols, bw, _, gsplit, gorder = data_wide
    assert gorder != sorted(gorder)   # the search picked a non-identity column order
    order = np.zeros(N_WIDE, np.uint32)
    group = np.zeros(N_WIDE, np.uint32)
    ng = ctx.run_plan(cols, bw, gsplit, order, group, col_order=gorder, hash=True)
    o, g, n_ref = O.run_plan_hash(cols, bw, gsplit, col_order=gorder)
    assert ng == n_ref
    assert np.array_equal(order, o)
    assert np.array_equal(group, g)


def test_4096_instances_sampled_vs_oracle(ctx):
    import torch

    from fastmulticolsort_b200 import batch_bench as BB
    cols, sizes, bw, split, _ = BB.instance_workload(torch)
    total = int(sizes.sum())
    order = torch.empty(total, dtype=torch.int32, device="cuda")
    group = torch.empty(total, dtype=torch.int32, device="cuda")
    counts = ctx.run_batch(cols, bw, split, sizes, order, group)
    ctx.synchronize()
    ok, bad = BB.check_instances_vs_oracle(cols, sizes, bw, split, order, group, counts,
                                           BB.sample_instances(sizes, count=20))
    assert ok, f"instance {bad} differs from the oracle"
    # the whole batch equals the same plan run instance by instance
    order2 = torch.empty_like(order)
    group2 = torch.empty_like(group)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for i in range(len(sizes)):
        a, b = int(offs[i]), int(offs[i + 1])
        ng = ctx.run_plan([c[a:b] for c in cols], bw, split, order2[a:b], group2[a:b])
        assert ng == int(counts[i]), i
    ctx.synchronize()
    assert torch.equal(order, order2)
    assert torch.equal(group, group2)
