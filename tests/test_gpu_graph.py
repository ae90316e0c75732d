"""fmcs_graph: a sort plan captured once as a CUDA graph and replayed on the
same device buffers, refilled between launches.  Exact parity with the
oracle on every replay."""
import numpy as np
import pytest

from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(a.view({2: np.int16, 4: np.int32, 8: np.int64}[a.dtype.itemsize])).cuda()


@pytest.mark.parametrize("kind,split", [("17b33", [50]), ("17b33", [17, 33]), ("17b33", [6, 44]),
                                        ("zipf", [20, 24, 40]), ("zipf", [44, 40])])
def test_graph_replays_match_oracle(ctx, kind, split):
    torch = pytest.importorskip("torch")
    n = 1 << 20
    make = (lambda s: W.cols_17b33(n, seed_index=s)) if kind == "17b33" else (lambda s: W.cols_zipf(n, seed_index=s))
    cols, bw = make(300)
    dcols = [_dev(torch, c) for c in cols]
    order = torch.zeros(n, dtype=torch.int32, device="cuda")
    group = torch.zeros(n, dtype=torch.int32, device="cuda")
    g = ctx.plan_graph(dcols, bw, split, order, group)
    try:
        for seed in (300, 300, 301):
            if seed != 300:
                cols, _ = make(seed)
                for d, c in zip(dcols, cols):
                    d.copy_(_dev(torch, c))
            torch.cuda.synchronize()
            ng = g.launch()
            o, gr, ng_ref = O.run_plan_sort(cols, bw, split)
            assert ng == ng_ref
            assert np.array_equal(order.cpu().numpy().view(np.uint32), o)
            assert np.array_equal(group.cpu().numpy().view(np.uint32), gr)
    finally:
        g.close()


def test_graph_level_loop_follows_the_data(ctx):
    """The radix levels of a captured plan run as a loop on the device: a
    replay on data that needs more levels than the captured run (constant
    and low-cardinality keys keep whole-array segments large level after
    level) or fewer (all keys distinct) still matches the oracle."""
    torch = pytest.importorskip("torch")
    n = 1 << 20
    widths, split = [20, 30], [50]
    datasets = [
        W.cols_uniform(n, widths, seed_index=310)[0],                       # captured on this
        [np.zeros(n, np.uint32), np.zeros(n, np.uint32)],                   # every level skips
        W.cols_uniform(n, widths, seed_index=311, distinct=[3, 5])[0],      # few distinct keys
        W.cols_uniform(n, widths, seed_index=312)[0],
        [np.full(n, 7, np.uint32), np.arange(n, dtype=np.uint32)[::-1].copy()],  # reverse order
    ]
    dcols = [_dev(torch, c) for c in datasets[0]]
    order = torch.zeros(n, dtype=torch.int32, device="cuda")
    group = torch.zeros(n, dtype=torch.int32, device="cuda")
    g = ctx.plan_graph(dcols, widths, split, order, group)
    try:
        assert g.kernels() > 0
        for cols in datasets:
            for d, c in zip(dcols, cols):
                d.copy_(_dev(torch, c))
            torch.cuda.synchronize()
            ng = g.launch()
            o, gr, ng_ref = O.run_plan_sort(cols, widths, split)
            assert ng == ng_ref
            assert np.array_equal(order.cpu().numpy().view(np.uint32), o)
            assert np.array_equal(group.cpu().numpy().view(np.uint32), gr)
    finally:
        g.close()


@pytest.mark.parametrize("widths,distinct,split,col_order", [
    ([8, 12, 7], [16, 300, 0], [27], None),
    ([8, 12, 7], [16, 300, 0], [8, 19], [0, 2, 1]),
    ([2, 1, 12, 12, 32, 7], [3, 2, 2526, 2526, 0, 100], [58, 8], [0, 2, 3, 4, 1, 5]),
    ([8, 8, 8], [4, 5, 6], [8, 8, 8], None),
])
def test_hash_graph_replays_match_oracle(ctx, widths, distinct, split, col_order):
    """A hash-grouping plan captured as a graph (fmcs_graph_create_hash): its
    key widths and its clustering are decided on the device, so replays on
    new data match the oracle's hash plan (src/composer.cpp:137-227)."""
    torch = pytest.importorskip("torch")
    n = 300_000
    cols, bw = W.cols_uniform(n, widths, seed_index=40, distinct=distinct)
    dcols = [_dev(torch, c) for c in cols]
    order = torch.zeros(n, dtype=torch.int32, device="cuda")
    group = torch.zeros(n, dtype=torch.int32, device="cuda")
    g = ctx.plan_graph(dcols, bw, split, order, group, col_order=col_order, hash=True)
    try:
        for seed in (40, 41, 40):
            cols, _ = W.cols_uniform(n, widths, seed_index=seed, distinct=distinct)
            for d, c in zip(dcols, cols):
                d.copy_(_dev(torch, c))
            torch.cuda.synchronize()
            ng = g.launch()
            o, gr, ng_ref = O.run_plan_hash(cols, bw, split, col_order=col_order)
            assert ng == ng_ref
            assert np.array_equal(order.cpu().numpy().view(np.uint32), o)
            assert np.array_equal(group.cpu().numpy().view(np.uint32), gr)
            # the same plan through the eager C ABI agrees
            oe = np.zeros(n, np.uint32)
            ge = np.zeros(n, np.uint32)
            assert ctx.run_plan(cols, bw, split, oe, ge, col_order=col_order, hash=True) == ng_ref
            assert np.array_equal(oe, o) and np.array_equal(ge, gr)
    finally:
        g.close()


def test_eager_round_skips_empty_tiers(ctx):
    """An eager sort round launches only the on-chip tiers its segments use:
    a round-0 sort of 1,000 rows is one block sort (and the group ids)."""
    rng = np.random.default_rng(5)
    n = 1000
    bank = rng.integers(0, 1 << 40, size=n, dtype=np.uint64)
    order = np.zeros(n, np.uint32)
    ctx.profile(True)
    ctx.sort_round(bank, 40, order)
    prof = ctx.profile_report()
    ctx.profile(False)
    ran = {k for k in prof if not k.startswith("_")}
    assert "block_sort_1024" in ran
    assert not ran & {"thread_sort", "warp_sort", "block_sort_512", "block_sort_2048", "block_sort_4096",
                      "block_sort_8192", "copy", "copy_tiles"}
    o_ref, _, _, _ = O.sort_round(bank)
    assert np.array_equal(order, o_ref)
