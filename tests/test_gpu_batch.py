"""fmcs_run_batch: many independent instances in one batch, each checked
against the oracle on its own rows (instance-local oids and group ids)."""
import numpy as np
import pytest

from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("split", [[8, 24, 40], [32, 40], [8, 64]])
def test_batch_matches_per_instance_oracle(ctx, split):
    rng = np.random.default_rng(sum(split))
    sizes = [1, 2, 3, 17, 129, 5000, 70000, 0, 1024, 4097, 12345, 1]
    sizes += list((2 ** rng.uniform(10, 16, size=20)).astype(int))
    total = int(sum(sizes))
    cols, bw = W.cols_uniform(total, [8, 24, 40], seed_index=5, distinct=[16, 0, 0])
    order = np.zeros(total, np.uint32)
    group = np.zeros(total, np.uint32)
    counts = ctx.run_batch(cols, bw, split, sizes, order, group)
    off = 0
    for k, n in enumerate(sizes):
        if n == 0:
            assert counts[k] == 0
            continue
        sub = [c[off:off + n].copy() for c in cols]
        o, g, ng = O.run_plan_sort(sub, bw, split)
        assert np.array_equal(order[off:off + n], o), k
        assert np.array_equal(group[off:off + n], g), k
        assert counts[k] == ng
        off += n


def test_batch_rejects_bad_instances(ctx):
    from fastmulticolsort_b200 import capi
    import ctypes
    cols, bw = W.cols_uniform(100, [8, 24], seed_index=6)
    L = capi.load()
    inst = (capi.Instance * 2)(capi.Instance(0, 50), capi.Instance(60, 40))   # gap: not contiguous
    ptrs = (ctypes.c_void_p * 2)(*[c.ctypes.data for c in cols])
    order = np.zeros(100, np.uint32)
    rc = L.fmcs_run_batch(ctx.handle, ptrs, capi._u32arr([2, 4]), capi._u32arr(bw), 2, capi._u32arr([32]), 1,
                          inst, 2, 100, order.ctypes.data, None, None)
    assert rc == capi.FMCS_E_INVAL
