"""The group-boundary scan (dense group ids of sorted keys, optionally within
the runs of a previous round's group ids) on every key width, at sizes on
and around the kernel's chunk and tile edges, with 16-byte-aligned and
misaligned arrays (vector and scalar loads).

Called through fmcs_group_ids_noalloc (the scan's count and prefix passes, its
id pass recomputing the boundary masks from the keys) and through a context's
sort round (the id pass reading the masks that the count pass kept); the
expected ids are the oracle's (extractGroupInfo, src/composer.cpp:630-678,
restated in oracle/fmcs_oracle.c) for keys that are already in order, so that
its stable sort leaves them in place.  Integer ids: the comparison is exact."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# tile counts (8,192 rows a tile) odd and even, among them 5 and 25 tiles: the
# workspace's sub-arrays start on 256-byte boundaries whatever the tile count
SIZES = [1, 2, 33, 1000, 8191, 8192, 8193, 40_960, 70_001, 200_000, 1_000_003]


def _as_int(a):
    return a.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[a.dtype.itemsize])


def _case(n, dtype, segmented, seed):
    """Keys in order within each run of in_group (or overall), with repeats."""
    rng = np.random.default_rng(seed)
    hi = min(int(np.iinfo(dtype).max), max(2, n // 8))
    keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(dtype)
    ig = None
    if segmented:
        starts = np.zeros(n, np.uint32)
        starts[rng.integers(0, n, size=max(1, n // 500))] = 1
        starts[0] = 0
        ig = np.cumsum(starts).astype(np.uint32)
        keys = keys[np.lexsort((keys, ig))]
    else:
        keys = np.sort(keys)
    return keys, ig


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.uint32, np.uint64])
@pytest.mark.parametrize("segmented", [False, True])
@pytest.mark.parametrize("misaligned", [False, True])
def test_boundary_scan_matches_oracle(dtype, segmented, misaligned):
    torch = pytest.importorskip("torch")
    from fastmulticolsort_b200 import capi

    def dev(a):
        # a misaligned view starts one element into its buffer, so that its
        # address is not 16-byte aligned (the scalar-load path)
        if not misaligned:
            return torch.from_numpy(_as_int(a)).cuda()
        return torch.from_numpy(_as_int(np.concatenate([a[:1], a]))).cuda()[1:]

    for n in SIZES:
        keys, ig = _case(n, dtype, segmented, seed=n * 7 + np.dtype(dtype).itemsize)
        _, g_ref, _, ng_ref = O.sort_round(keys, order=np.arange(n, dtype=np.uint32), in_group=ig)
        kd = dev(keys)
        igd = None if ig is None else dev(ig)
        outv = dev(np.full(n, 0xFFFFFFFF, np.uint32))
        ng = capi.group_ids_noalloc(kd, outv, in_group=igd)
        torch.cuda.synchronize()
        got = outv.cpu().numpy().view(np.uint32)
        assert ng == ng_ref, (n, ng, ng_ref)
        assert np.array_equal(got, g_ref), n


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32, np.uint64])
@pytest.mark.parametrize("segmented", [False, True])
@pytest.mark.parametrize("misaligned", [False, True])
def test_sort_round_group_ids_of_ordered_keys(dtype, segmented, misaligned):
    """The same sweep through a context's sort round (whose scan keeps the
    boundary masks of its first pass in the workspace): keys already in order
    stay in place, and the group ids are the scan's.  Misaligned: the caller's
    in_group and group arrays start one element into their buffers, so the
    scans that read or write them take their scalar paths."""
    torch = pytest.importorskip("torch")
    from fastmulticolsort_b200 import capi

    def dev(a):
        if not misaligned:
            return torch.from_numpy(_as_int(a)).cuda()
        return torch.from_numpy(_as_int(np.concatenate([a[:1], a]))).cuda()[1:]

    with capi.Context(0) as ctx:
        for n in SIZES[1:]:
            keys, ig = _case(n, dtype, segmented, seed=n * 11 + np.dtype(dtype).itemsize)
            o_ref, g_ref, _, ng_ref = O.sort_round(keys, order=np.arange(n, dtype=np.uint32), in_group=ig)
            kd = torch.from_numpy(_as_int(keys)).cuda()
            igd = None if ig is None else dev(ig)
            order = torch.arange(n, dtype=torch.int32, device="cuda")
            grp = dev(np.full(n, 0xFFFFFFFF, np.uint32))
            ng = ctx.sort_round(kd, 8 * np.dtype(dtype).itemsize, order, in_group=igd, out_group=grp)
            torch.cuda.synchronize()
            assert ng == ng_ref, (n, ng, ng_ref)
            assert np.array_equal(order.cpu().numpy().view(np.uint32), o_ref), n
            assert np.array_equal(grp.cpu().numpy().view(np.uint32), g_ref), n
