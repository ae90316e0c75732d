"""The serving loop (include/fmcs_server.h): each request's result is the same
when it runs alone and when it runs in a mix of concurrent requests that
overlap on the device and share batched launches; admission keeps the
admitted footprint within the HBM budget.  Integer results: exact."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_requests(torch, count=24, seed=3):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(2 ** rng.uniform(10, 20)) if i % 3 else int(2 ** rng.uniform(20, 22))
        widths = [8, 24, 40] if i % 2 else [17, 33]
        cols, bw = W.cols_uniform(n, widths, seed_index=100 + i, distinct=[16] + [0] * (len(widths) - 1))
        dcols = [torch.from_numpy(c.view({2: np.int16, 4: np.int32, 8: np.int64}[c.dtype.itemsize])).cuda()
                 for c in cols]
        split = None if i % 4 == 0 else ([sum(widths) - 40, 40] if i % 2 else [50])
        reqs.append(dict(cols=cols, dcols=dcols, bw=bw, n=n, split=split, hash=(i % 5 == 4)))
    return reqs


def run(server, torch, reqs, together):
    outs = []
    tickets = []
    for r in reqs:
        o = torch.full((r["n"],), -1, dtype=torch.int32, device="cuda")
        g = torch.full((r["n"],), -1, dtype=torch.int32, device="cuda")
        outs.append((o, g))
        t = server.submit(r["dcols"], r["bw"], o, g, split=r["split"], hash=r["hash"])
        if together:
            tickets.append(t)
        else:
            res = server.wait(t)
            assert res["status"] == 0
            tickets.append(res)
    results = [server.wait(t) for t in tickets] if together else tickets
    for res in results:
        assert res["status"] == 0
    return [(o.cpu().numpy().view(np.uint32), g.cpu().numpy().view(np.uint32)) for o, g in outs], results


def test_same_alone_and_in_the_mix():
    torch = pytest.importorskip("torch")
    reqs = make_requests(torch)
    with capi.Server(0, hbm_budget_bytes=40 << 30, slots=4, batch_rows_max=1 << 20) as srv:
        alone, _ = run(srv, torch, reqs, together=False)
        mixed, _ = run(srv, torch, reqs, together=True)        # four slots: work overlaps
    with capi.Server(0, hbm_budget_bytes=40 << 30, slots=1, batch_rows_max=1 << 20) as srv:
        queued, results = run(srv, torch, reqs, together=True)  # one slot: requests queue and batch
    for k in range(len(reqs)):
        assert np.array_equal(alone[k][0], mixed[k][0]) and np.array_equal(alone[k][1], mixed[k][1]), k
        assert np.array_equal(alone[k][0], queued[k][0]) and np.array_equal(alone[k][1], queued[k][1]), k
    assert max(r["batched_with"] for r in results) > 1   # small requests shared launches
    # and the results are the reference's (the oracle's)
    for k in (1, 2, 5):
        r = reqs[k]
        if r["hash"]:
            continue
        o, g, _ = O.run_plan_sort(r["cols"], r["bw"], r["split"])
        assert np.array_equal(alone[k][0], o) and np.array_equal(alone[k][1], g)


def test_admission_respects_the_budget():
    torch = pytest.importorskip("torch")
    reqs = make_requests(torch, count=10, seed=9)
    budget = 600 << 20   # room for a few requests at a time
    with capi.Server(0, hbm_budget_bytes=budget, slots=4, batch_rows_max=0) as srv:
        tickets = []
        peak = 0
        for r in reqs:
            o = torch.empty(r["n"], dtype=torch.int32, device="cuda")
            tickets.append((srv.submit(r["dcols"], r["bw"], o, split=r["split"]), o))
            peak = max(peak, srv.load()[0])
        for t, _ in tickets:
            assert srv.wait(t)["status"] == 0
            peak = max(peak, srv.load()[0])
        assert peak <= budget
        # a request larger than the whole budget is refused up front
        big = torch.empty(40_000_000, dtype=torch.int64, device="cuda")
        with pytest.raises(capi.FmcsError) as e:
            srv.submit([big], [40], torch.empty(40_000_000, dtype=torch.int32, device="cuda"), split=[40])
        assert e.value.code == capi.FMCS_E_OOM
