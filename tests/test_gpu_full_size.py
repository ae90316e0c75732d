"""Full-size workloads (16,777,216 rows of 17/33-bit codes) through the C ABI:
size-independent properties (sortedness of the key tuples, permutation,
group ids consistent with the keys) for every bit-borrowing plan, and
bit-exact parity with the oracle for the headline plans."""
import numpy as np
import pytest

from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 16_777_216


@pytest.fixture(scope="module")
def data():
    return W.cols_17b33(N)


def check_properties(cols, order, group):
    n = order.shape[0]
    assert np.array_equal(np.sort(order), np.arange(n, dtype=np.uint32))   # permutation
    k0 = cols[0][order].astype(np.uint64)
    k1 = cols[1][order]
    key = (k0 << np.uint64(33)) | k1
    d = np.diff(key.astype(np.uint64))
    assert np.all(key[1:] >= key[:-1])                                      # sorted tuples
    new = key[1:] != key[:-1]
    assert np.array_equal(np.diff(group.astype(np.int64)), new.astype(np.int64))   # dense ids
    ties = ~new
    assert np.all(order[1:][ties] > order[:-1][ties])                        # canonical ties
    del d


@pytest.mark.parametrize("k", list(range(0, 18)))
def test_bit_borrowing_plans_properties(ctx, data, k):
    cols, bw = data
    split = W.split_for_k(k)
    order = np.zeros(N, np.uint32)
    group = np.zeros(N, np.uint32)
    ctx.run_plan(cols, bw, split, order, group)
    check_properties(cols, order, group)


@pytest.mark.slow
@pytest.mark.parametrize("split", [[50], [17, 33]])
def test_full_size_parity(ctx, data, split):
    cols, bw = data
    order = np.zeros(N, np.uint32)
    group = np.zeros(N, np.uint32)
    ng = ctx.run_plan(cols, bw, split, order, group)
    o_ref, g_ref, ng_ref = O.run_plan_sort(cols, bw, split)
    assert ng == ng_ref
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, g_ref)
