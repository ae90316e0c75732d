"""Edge cases through the C ABI: empty inputs (every entry point returns OK
and writes nothing), one row, a row count at the 32-bit oid limit (rejected
on the host before any device work), and the tiny sizes just around the
on-chip tiers' capacities, all against the oracle.  The reference's own tests
are randomized property checks over such shapes (tests/*_test.cpp)."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_empty_inputs(ctx):
    e32 = np.zeros(0, np.uint32)
    e64 = np.zeros(0, np.uint64)
    assert ctx.run_plan([e32, e64], [17, 33], [50], e32.copy(), e32.copy()) == 0
    assert ctx.run_plan([e32, e64], [17, 33], [17, 33], e32.copy(), e32.copy(), hash=True) == 0
    assert ctx.sort_round(e64, 40, e32.copy(), out_group=e32.copy()) == 0
    assert ctx.hash_round(e64, e32.copy(), out_group=e32.copy()) == 0
    ctx.gather(e64, e32, e64.copy())
    ctx.stitch([(e32, 17, 1, 17)], e64.copy())
    counts = ctx.run_batch([e32, e64], [17, 33], [50], [0, 0, 0], e32.copy(), e32.copy())
    assert list(counts) == [0, 0, 0]


@pytest.mark.parametrize("split", [[50], [17, 33]])
def test_one_row(ctx, split):
    cols = [np.array([12345], np.uint32), np.array([987654321], np.uint64)]
    order = np.full(1, 7, np.uint32)
    group = np.full(1, 7, np.uint32)
    assert ctx.run_plan(cols, [17, 33], split, order, group) == 1
    assert order[0] == 0 and group[0] == 0


def test_row_count_limit_rejected(ctx):
    """n >= 2^32 does not fit a 32-bit oid: FMCS_E_INVAL from the host checks
    (the arrays are never touched, so tiny stand-ins suffice)."""
    import ctypes
    L = capi.load()
    a = np.zeros(4, np.uint64)
    o = np.zeros(4, np.uint32)
    ng = ctypes.c_uint32(0)
    rc = L.fmcs_sort_round(ctx.handle, a.ctypes.data, 8, 40, o.ctypes.data, None, None, None, 1 << 32,
                           ctypes.byref(ng))
    assert rc == capi.FMCS_E_INVAL


def test_hash_row_limit_rejected(ctx):
    """Hash rounds take n < 2^31 (32-bit slot indices below two sentinels):
    FMCS_E_INVAL before any staging (tiny stand-in arrays)."""
    import ctypes
    L = capi.load()
    a = np.zeros(4, np.uint64)
    o = np.zeros(4, np.uint32)
    g = np.zeros(4, np.uint32)
    ng = ctypes.c_uint32(0)
    rc = L.fmcs_hash_round(ctx.handle, a.ctypes.data, 8, o.ctypes.data, None, g.ctypes.data, 1 << 31, 0,
                           ctypes.byref(ng))
    assert rc == capi.FMCS_E_INVAL
    rc = L.fmcs_hash_round_unordered(ctx.handle, a.ctypes.data, 8, None, g.ctypes.data, 1 << 31, ctypes.byref(ng))
    assert rc == capi.FMCS_E_INVAL


@pytest.mark.parametrize("n", [2, 15, 16, 17, 32, 33, 128, 129, 512, 513, 2048, 2049, 2304, 2305, 4096, 4097,
                               8192, 8193])
def test_tier_edges_round0(ctx, n):
    rng = np.random.default_rng(n)
    bank = rng.integers(0, 1 << 20, size=n, dtype=np.uint64)   # repeats at every size
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.sort_round(bank, 20, order, out_group=group)
    o, g, _, ng_ref = O.sort_round(bank)
    assert ng == ng_ref and np.array_equal(order, o) and np.array_equal(group, g)


def test_segments_at_every_tier_edge(ctx):
    """One segmented round whose segments sit on both sides of every tier's
    capacity, with keys that tie inside segments."""
    rng = np.random.default_rng(3)
    sizes = [1, 2, 15, 16, 17, 32, 33, 128, 129, 512, 513, 1024, 1025, 2048, 2049, 2304, 2305, 4096, 4097,
             8192, 8193, 20000]
    sizes = list(rng.permutation(sizes))
    n = int(sum(sizes))
    in_group = np.repeat(np.arange(len(sizes), dtype=np.uint32), sizes)
    bank = (rng.integers(0, 1 << 30, size=n, dtype=np.uint64) % 997).astype(np.uint32)
    order_in = rng.permutation(n).astype(np.uint32)
    order = order_in.copy()
    group = np.zeros(n, np.uint32)
    ng = ctx.sort_round(bank, 32, order, in_group=in_group, out_group=group)
    o, g, _, ng_ref = O.sort_round(bank, order=order_in, in_group=in_group)
    assert ng == ng_ref and np.array_equal(order, o) and np.array_equal(group, g)
