"""The allocation-free entry point fmcs_group_ids_noalloc, called through the
C ABI, against the group ids of the existing entry point fmcs_sort_round.

Callers that cannot let a library allocate device memory (engines that keep
all of HBM in their own pool, latency-critical callers that cannot take the
device-wide synchronization of cudaMalloc/cudaFree) use this entry point; its
scratch is a static device array of the library, shared by every call.  The
test makes two different calls in a row so that the second one runs on the
first one's leftover scratch.  Integer ids: the comparison is exact.  This
file is collected last so that a failure here stops a `-x` run only after
every other test has run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _segments(rng, n):
    sizes = rng.integers(1, 3000, size=n)
    cs = np.cumsum(sizes)
    cs = cs[cs < n]
    g = np.zeros(n, np.uint32)
    g[cs] = 1
    return np.cumsum(g).astype(np.uint32)


def _as_int(a):
    return a.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[a.dtype.itemsize])


def test_noalloc_matches_sort_round_group_ids():
    torch = pytest.importorskip("torch")
    from fastmulticolsort_b200 import capi

    cases = [
        (1_000_003, np.uint64, 40, False),   # round 0 shape
        (300_001, np.uint32, 20, True),      # later round: runs of in_group
        (4097, np.uint16, 9, True),
    ]
    with capi.Context(0) as ctx:
        for n, dtype, bits, segmented in cases:
            rng = np.random.default_rng(n)
            bank = rng.integers(0, 1 << (bits - 3), size=n, dtype=np.uint64).astype(dtype)
            bank_d = torch.from_numpy(_as_int(bank)).cuda()
            if segmented:
                ig = _segments(rng, n)
                ig_d = torch.from_numpy(_as_int(ig)).cuda()
                order_d = torch.from_numpy(_as_int(rng.permutation(n).astype(np.uint32))).cuda()
            else:
                ig_d = None
                order_d = torch.zeros(n, dtype=torch.int32, device="cuda")
            keys_d = torch.empty_like(bank_d)
            grp_d = torch.empty(n, dtype=torch.int32, device="cuda")
            # existing entry point: sorted keys and their group ids
            ng_ref = ctx.sort_round(bank_d, bits, order_d, in_group=ig_d, out_group=grp_d,
                                    sorted_bank=keys_d)
            out_d = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            ng = capi.group_ids_noalloc(keys_d, out_d, in_group=ig_d)
            torch.cuda.synchronize()
            assert ng == ng_ref
            assert torch.equal(out_d, grp_d)


def test_noalloc_rejects_what_it_cannot_do_without_allocating():
    torch = pytest.importorskip("torch")
    from fastmulticolsort_b200 import capi

    L = capi.load()
    keys = torch.zeros(16, dtype=torch.int64, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    import ctypes
    ng = ctypes.c_uint32(0)
    # beyond the static scratch (67,108,864 rows): rejected before any GPU work
    rc = L.fmcs_group_ids_noalloc(None, keys.data_ptr(), 8, None, out.data_ptr(), 67_108_865, ctypes.byref(ng))
    assert rc == capi.FMCS_E_INVAL
    # host memory would have to be staged through an allocation: rejected
    hk = np.zeros(16, np.uint64)
    ho = np.zeros(16, np.uint32)
    rc = L.fmcs_group_ids_noalloc(None, hk.ctypes.data, 8, None, ho.ctypes.data, 16, ctypes.byref(ng))
    assert rc == capi.FMCS_E_INVAL
