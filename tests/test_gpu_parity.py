"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference-generated golden fixtures.  Integer work: bit-exact."""
import numpy as np
import pytest

from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O
from tests.golden_util import case_id, digest, load_cases

pytestmark = pytest.mark.gpu

CASES = load_cases()


@pytest.mark.parametrize("c", CASES, ids=[case_id(c) for c in CASES])
def test_run_plan_matches_golden(ctx, c):
    n = c["n"]
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.run_plan(c["cols"], c["bw"], c["split"], order, group, hash=(c["path"] == "hash"))
    assert digest(order) == c["order_sha256"]
    assert digest(group) == c["group_sha256"]
    assert ng == c["ngroups"]


SIZES = [1, 2, 3, 31, 32, 33, 127, 128, 129, 1023, 1024, 1025, 4095, 4096, 4097, 8191, 8193,
         65536 + 7, 1 << 20]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype,bits", [(np.uint16, 11), (np.uint32, 17), (np.uint32, 32),
                                        (np.uint64, 50), (np.uint64, 64)])
def test_sort_round0(ctx, n, dtype, bits):
    rng = np.random.default_rng(n * 7 + bits)
    hi = (1 << bits) - 1
    bank = rng.integers(0, hi, size=n, dtype=np.uint64, endpoint=True).astype(dtype)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    keys = np.zeros(n, dtype)
    ng = ctx.sort_round(bank, bits, order, out_group=group, sorted_bank=keys)
    o_ref, g_ref, k_ref, ng_ref = O.sort_round(bank)
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, g_ref)
    assert np.array_equal(keys, k_ref)
    assert ng == ng_ref


@pytest.mark.parametrize("n", [5000, 70000, 1 << 20])
@pytest.mark.parametrize("distinct", [1, 3, 40, 2000])
def test_sort_round0_duplicates(ctx, n, distinct):
    rng = np.random.default_rng(n + distinct)
    pool = rng.integers(0, 1 << 40, size=distinct, dtype=np.uint64)
    bank = pool[rng.integers(0, distinct, size=n)]
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.sort_round(bank, 40, order, out_group=group)
    o_ref, g_ref, _, ng_ref = O.sort_round(bank)
    assert np.array_equal(order, o_ref) and np.array_equal(group, g_ref) and ng == ng_ref


def _segments(rng, n, kind):
    if kind == "uniform":
        sizes = rng.integers(1, 300, size=n)
    elif kind == "tiers":
        # straddle every tier threshold
        base = np.array([1, 2, 3, 15, 16, 17, 31, 32, 33, 127, 128, 129, 511, 512, 513, 1023, 1024, 1025,
                         2047, 2048, 2049, 4095, 4096, 4097, 9000, 70000])
        sizes = rng.permutation(np.repeat(base, 3))
    else:  # zipf-like
        sizes = np.maximum(1, (20000 / np.arange(1, 2000)).astype(np.int64))
        sizes = rng.permutation(sizes)
    cs = np.cumsum(sizes)
    cs = cs[cs <= n]
    grp = np.zeros(n, np.uint32)
    grp[cs[cs < n]] = 1
    return np.cumsum(grp).astype(np.uint32)


@pytest.mark.parametrize("kind", ["uniform", "tiers", "zipf"])
@pytest.mark.parametrize("dtype,bits", [(np.uint16, 16), (np.uint32, 24), (np.uint64, 40)])
def test_sort_round_segmented(ctx, kind, dtype, bits):
    rng = np.random.default_rng(hash((kind, bits)) & 0xFFFF)
    n = 300000
    in_group = _segments(rng, n, kind)
    order_in = rng.permutation(n).astype(np.uint32)
    bank = rng.integers(0, (1 << bits) - 1, size=n, dtype=np.uint64, endpoint=True).astype(dtype)
    if kind == "zipf":
        bank = (bank % 50).astype(dtype)   # many ties
    order = order_in.copy()
    group = np.zeros(n, np.uint32)
    keys = np.zeros(n, dtype)
    ng = ctx.sort_round(bank, bits, order, in_group=in_group, out_group=group, sorted_bank=keys)
    o_ref, g_ref, k_ref, ng_ref = O.sort_round(bank, order=order_in, in_group=in_group)
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, g_ref)
    assert np.array_equal(keys, k_ref)
    assert ng == ng_ref


@pytest.mark.parametrize("src_bytes,bank_bytes", [(2, 2), (2, 4), (4, 4), (4, 8), (8, 8), (1, 2), (8, 2),
                                                  (1, 1)])
@pytest.mark.parametrize("n", [1, 5, 4099])
def test_stitch(ctx, src_bytes, bank_bytes, n):
    rng = np.random.default_rng(src_bytes * 100 + bank_bytes + n)
    bits = 8 * src_bytes if src_bytes < 8 else 61
    a = rng.integers(0, 1 << min(bits, 62), size=n, dtype=np.uint64).astype(np.dtype(f"u{src_bytes}"))
    b = rng.integers(0, 1 << 5, size=n, dtype=np.uint64).astype(np.uint16)
    cap = 8 * bank_bytes
    w = min(bits, cap - 5)
    sl = [(b, 5, 1, 5), (a, bits, bits - w + 1, bits)]
    out = np.zeros(n, np.dtype(f"u{bank_bytes}"))
    ctx.stitch(sl, out)
    assert np.array_equal(out, O.stitch(sl, bank_bytes, n))


@pytest.mark.parametrize("bank_bytes", [1, 2, 4, 8])
def test_gather(ctx, bank_bytes):
    rng = np.random.default_rng(bank_bytes)
    n = 100003
    bank = rng.integers(0, 255, size=n, dtype=np.uint64).astype(np.dtype(f"u{bank_bytes}"))
    order = rng.permutation(n).astype(np.uint32)
    out = np.zeros(n, bank.dtype)
    ctx.gather(bank, order, out)
    assert np.array_equal(out, bank[order])


@pytest.mark.parametrize("bank_bytes,distinct", [(1, 50), (2, 3000), (4, 100000), (8, 7)])
@pytest.mark.parametrize("segmented", [False, True])
@pytest.mark.parametrize("last", [False, True])
def test_hash_round(ctx, bank_bytes, distinct, segmented, last):
    rng = np.random.default_rng(bank_bytes * 31 + distinct)
    n = 200000
    pool = rng.integers(0, 1 << (8 * bank_bytes - 1), size=distinct, dtype=np.uint64)
    bank = pool[rng.integers(0, distinct, size=n)].astype(np.dtype(f"u{bank_bytes}"))
    if segmented:
        in_group = _segments(rng, n, "uniform")
        order_in = rng.permutation(n).astype(np.uint32)
    else:
        in_group, order_in = None, None
    order = np.zeros(n, np.uint32) if order_in is None else order_in.copy()
    group = np.zeros(n, np.uint32)
    ng = ctx.hash_round(bank, order, in_group=in_group, out_group=group, last_round=last)
    o_ref, og_ref, idx_ref, ng_ref = O.hash_round(bank, order=order_in, in_group=in_group, last_round=last)
    assert ng == ng_ref
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, idx_ref if last else og_ref)


def test_device_pointers(ctx):
    torch = pytest.importorskip("torch")
    cols, bw = W.cols_17b33(1 << 18, seed_index=31)
    dcols = [torch.from_numpy(c.view(np.int32) if c.dtype == np.uint32 else c.view(np.int64)).cuda()
             for c in cols]
    order = torch.zeros(cols[0].shape[0], dtype=torch.int32, device="cuda")
    group = torch.zeros_like(order)
    ng = ctx.run_plan(dcols, bw, [50], order, group)
    o_ref, g_ref, ng_ref = O.run_plan_sort(cols, bw, [50])
    assert ng == ng_ref
    assert np.array_equal(order.cpu().numpy().view(np.uint32), o_ref)
    assert np.array_equal(group.cpu().numpy().view(np.uint32), g_ref)


def test_invalid_arguments(ctx):
    from fastmulticolsort_b200 import capi
    bank = np.zeros(10, np.uint64)
    order = np.zeros(10, np.uint32)
    with pytest.raises(capi.FmcsError) as e:
        ctx.sort_round(bank, 0, order)
    assert e.value.code == capi.FMCS_E_INVAL
    with pytest.raises(capi.FmcsError):
        ctx.sort_round(bank, 65, order)
    with pytest.raises(capi.FmcsError):
        ctx.run_plan([np.zeros(10, np.uint32), np.zeros(10, np.uint64)], [17, 33], [40], order)
    # the context keeps working after errors
    ng = ctx.sort_round(np.arange(10, dtype=np.uint64)[::-1].copy(), 8, order, out_group=np.zeros(10, np.uint32))
    assert ng == 10 and list(order) == list(range(9, -1, -1))


@pytest.mark.parametrize("bank_bytes", [1, 2, 4, 8])
def test_shift_left_and_assemble(ctx, bank_bytes):
    rng = np.random.default_rng(bank_bytes + 100)
    n = 70001
    dt = np.dtype(f"u{bank_bytes}")
    bank = rng.integers(0, 255, size=n, dtype=np.uint64).astype(dt)
    src = rng.integers(0, 1 << 20, size=n, dtype=np.uint64).astype(np.uint32)
    b = bank.copy()
    ctx.shift_left(b, 3)
    assert np.array_equal(b, (bank.astype(np.uint64) << np.uint64(3)).astype(dt))
    ctx.assemble(b, src, 20, 18, 20)   # the low 3 bits of a 20-bit column
    exp = ((bank.astype(np.uint64) << np.uint64(3)) | (src.astype(np.uint64) & np.uint64(7))).astype(dt)
    assert np.array_equal(b, exp)


@pytest.mark.parametrize("bank_bytes,distinct", [(1, 30), (4, 5000), (8, 100000)])
def test_hash_round_unordered(ctx, bank_bytes, distinct):
    from fastmulticolsort_b200 import capi
    rng = np.random.default_rng(distinct)
    n = 150000
    pool = rng.integers(0, 1 << (8 * bank_bytes - 1), size=distinct, dtype=np.uint64)
    bank = pool[rng.integers(0, distinct, size=n)].astype(np.dtype(f"u{bank_bytes}"))
    prev = rng.integers(0, 40, size=n, dtype=np.uint32)
    for ig in (None, prev):
        out = np.zeros(n, np.uint32)
        ng = C_hash_unordered(ctx, bank, ig, out)
        ref, ng_ref = O.hash_unordered(bank, ig)
        assert ng == ng_ref and np.array_equal(out, ref)


def C_hash_unordered(ctx, bank, in_group, out):
    import ctypes
    from fastmulticolsort_b200 import capi
    L = capi.load()
    L.fmcs_hash_round_unordered.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]
    ng = ctypes.c_uint32(0)
    rc = L.fmcs_hash_round_unordered(ctx.handle, bank.ctypes.data, bank.dtype.itemsize,
                                     None if in_group is None else in_group.ctypes.data, out.ctypes.data,
                                     bank.shape[0], ctypes.byref(ng))
    assert rc == 0
    return ng.value


@pytest.mark.parametrize("segmented", [False, True])
@pytest.mark.parametrize("dtype,bits", [(np.uint32, 24), (np.uint64, 40)])
def test_sort_round_plain(ctx, segmented, dtype, bits):
    rng = np.random.default_rng(bits + segmented)
    n = 250001
    bank = rng.integers(0, (1 << bits) - 1, size=n, dtype=np.uint64, endpoint=True).astype(dtype)
    bank[::7] = bank[3]   # ties
    if segmented:
        in_group = _segments(rng, n, "zipf")
        order_in = rng.permutation(n).astype(np.uint32)
    else:
        in_group, order_in = None, None
    order = np.zeros(n, np.uint32) if order_in is None else order_in.copy()
    group = np.zeros(n, np.uint32)
    keys = np.zeros(n, dtype)
    ng = ctx.sort_round_plain(bank, bits, order, in_group=in_group, out_group=group, sorted_bank=keys)
    o_ref, g_ref, k_ref, ng_ref = O.sort_round(bank, order=order_in, in_group=in_group)
    assert np.array_equal(order, o_ref) and np.array_equal(group, g_ref) and np.array_equal(keys, k_ref)
    assert ng == ng_ref


@pytest.mark.parametrize("knobs", [dict(rank_mode=0), dict(rank_mode=1), dict(rank_mode=2), dict(local_max=1024),
                                   dict(local_max=2048, msd_items=16), dict(msd_items=16, rank_mode=1),
                                   dict(msd_items=8, rank_mode=2), dict(local_max=8192)])
def test_tuning_knobs_same_results(knobs):
    from fastmulticolsort_b200 import capi
    cols, bw = W.cols_zipf(400000, seed_index=77)
    with capi.Context(0) as c:
        for k, v in knobs.items():
            c.set_tuning(k, v)
            assert c.get_tuning(k) == v
        for split in ([20, 24, 40], [44, 40]):
            order = np.zeros(400000, np.uint32)
            group = np.zeros(400000, np.uint32)
            ng = c.run_plan(cols, bw, split, order, group)
            o, g, n_ref = O.run_plan_sort(cols, bw, split)
            assert ng == n_ref and np.array_equal(order, o) and np.array_equal(group, g)
        with pytest.raises(capi.FmcsError):
            c.set_tuning("local_max", 9000)
        with pytest.raises(capi.FmcsError):
            c.set_tuning("rank_mode", 3)


@pytest.mark.parametrize("local_max", [4096, 8192])
@pytest.mark.parametrize("dtype,bits", [(np.uint32, 32), (np.uint64, 64)])
def test_sort_round_block_tier_key_shapes(dtype, bits, local_max):
    """Segments of every block tier (129..8192 rows) whose keys are distinct,
    repeated up to exactly 64 and 65 times (the largest bucket the rank-by-
    counting path takes, and one more), constant, differing only in the top
    or only in the lowest bit, and in reverse order: the stable order of the
    oracle in every case."""
    rng = np.random.default_rng(bits)
    segs = []
    for length in (129, 512, 513, 1024, 1025, 2048, 2049, 4096, 4097, 8192):
        top = (1 << (bits - 1))
        shapes = [
            rng.integers(0, (1 << bits) - 1, size=length, dtype=np.uint64, endpoint=True),
            np.repeat(rng.integers(0, 1 << 20, size=length // 64 + 1, dtype=np.uint64), 64)[:length],
            np.repeat(rng.integers(0, 1 << 20, size=length // 65 + 1, dtype=np.uint64), 65)[:length],
            np.full(length, 12345, np.uint64),
            (rng.integers(0, 2, size=length, dtype=np.uint64) * top) | 5,
            rng.integers(0, 2, size=length, dtype=np.uint64) | (top - 2),
            np.arange(length, dtype=np.uint64)[::-1] * 977,
        ]
        for sh in shapes:
            segs.append(rng.permutation(sh).astype(dtype))
    by_position = np.concatenate(segs)
    n = by_position.shape[0]
    sizes = [s.shape[0] for s in segs]
    in_group = np.repeat(np.arange(len(sizes), dtype=np.uint32), sizes)
    order_in = rng.permutation(n).astype(np.uint32)
    bank = np.empty_like(by_position)
    bank[order_in] = by_position          # position i of the round holds by_position[i]
    order = order_in.copy()
    group = np.zeros(n, np.uint32)
    keys = np.zeros(n, dtype)
    from fastmulticolsort_b200 import capi
    with capi.Context(0) as c:
        c.set_tuning("local_max", local_max)
        ng = c.sort_round(bank, bits, order, in_group=in_group, out_group=group, sorted_bank=keys)
    o_ref, g_ref, k_ref, ng_ref = O.sort_round(bank, order=order_in, in_group=in_group)
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, g_ref)
    assert np.array_equal(keys, k_ref)
    assert ng == ng_ref


@pytest.mark.parametrize("desc", [[True, False], [False, True], [True, True]])
@pytest.mark.parametrize("split", [[17, 33], [50], [6, 44]])
def test_run_plan_descending_columns(ctx, desc, split):
    """A descending column sorts like the ascending sort of (2^bw - 1 - value)
    (its bits inverted inside the declared width): parity with the oracle run
    on the inverted columns, ties in ascending oid as everywhere."""
    n = 300000
    cols, bw = W.cols_17b33(n, seed_index=41)
    inv = [((np.uint64(1) << np.uint64(w)) - np.uint64(1) - c.astype(np.uint64)).astype(c.dtype) if d else c
           for c, w, d in zip(cols, bw, desc)]
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.run_plan(cols, bw, split, order, group, descending=desc)
    o_ref, g_ref, ng_ref = O.run_plan_sort(inv, bw, split)
    assert ng == ng_ref
    assert np.array_equal(order, o_ref)
    assert np.array_equal(group, g_ref)
    # the keys really descend: the first column's values along the order
    v0 = cols[0][order].astype(np.int64)
    d0 = np.diff(v0)
    assert (d0 <= 0).all() if desc[0] else (d0 >= 0).all()


@pytest.mark.parametrize("hash_path", [False, True])
def test_group_by_column_order_matches_oracle(ctx, hash_path):
    """GROUP BY may reorder the columns (the optimizer's ordered=0 search,
    src/stitch_composer.cpp:15-35, 3877-3882): the column order it picks for
    the wide shape is not the identity, and the plan run with that order
    (sort or hash rounds) matches the oracle given the same order."""
    from fastmulticolsort_b200 import capi
    n = 400_000
    widths, distinct = [2, 1, 12, 12, 32, 7], [3, 2, 2526, 2526, 0, 100]
    cols, bw = W.cols_uniform(n, widths, seed_index=17, distinct=distinct)
    # the search on the 60,000,000-row table's statistics (at this row count
    # the identity order is already the cheapest)
    card = [k if k else 60_000_000 for k in distinct]
    split, corder, _ = capi.optimize_plan(bw, card, [c.dtype.itemsize for c in cols], 60_000_000, ordered=False)
    assert corder != sorted(corder)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.run_plan(cols, bw, split, order, group, col_order=corder, hash=hash_path)
    run = O.run_plan_hash if hash_path else O.run_plan_sort
    o, g, ng_ref = run(cols, bw, split, col_order=corder)
    assert ng == ng_ref
    assert np.array_equal(order, o) and np.array_equal(group, g)
