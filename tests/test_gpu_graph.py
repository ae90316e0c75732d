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
