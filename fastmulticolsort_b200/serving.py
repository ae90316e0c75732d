"""Serving benchmark: a trace of multi-column sort requests through the
serving loop (include/fmcs_server.h), against serial plain execution.

Workload (seeded): Poisson arrivals at `rate` requests/s; each request has a
row count log-uniform in [65,536, 67,108,864] and 2-6 columns of 1-64 bits
(sum <= 192) whose codes are uniform or Zipf(0.8); columns are generated on
the device and stay resident.  Requests draw their data from a pool of
`pool` pre-generated datasets.

Served:  fmcs_server with the cost model's plan per request, `slots`
         overlapping execution slots, admission against the HBM budget and
         continuous batching of small requests.
Serial plain: the same trace, one request at a time, one full-array sort per
         original column (fmcs_sort_round_plain); latency = completion -
         arrival on a timeline where a request starts when the previous one
         is done.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import capi

MIN_ROWS, MAX_ROWS = 1 << 16, 1 << 26


def _zipf_codes(torch, rng, n, w, s=0.8):
    k = min(1 << min(w, 62), 1 << 20)
    ranks = torch.arange(1, k + 1, dtype=torch.float64, device="cuda")
    cdf = torch.cumsum(ranks.pow(-s), 0)
    cdf /= cdf[-1].clone()
    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(1 << 62)))
    u = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    r = torch.searchsorted(cdf, u).clamp_(max=k - 1)
    codes = torch.from_numpy(rng.integers(0, 1 << min(w, 62), size=k, dtype=np.int64)).cuda()
    if w == 64:
        codes = codes * 2 + torch.from_numpy(rng.integers(0, 2, size=k, dtype=np.int64)).cuda()
    return codes[r]


def _uniform_codes(torch, rng, n, w):
    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(1 << 62)))
    if w == 64:
        return torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64, device="cuda", generator=g)
    if w == 63:
        return torch.randint(0, (1 << 63) - 1, (n,), dtype=torch.int64, device="cuda", generator=g)
    return torch.randint(0, 1 << w, (n,), dtype=torch.int64, device="cuda", generator=g)


def _store(torch, v, w):
    """Unsigned codes of w bits in the reference's storage width (u16/u32/u64),
    as the signed torch dtype of the same size and bits."""
    if w > 32:
        return v.contiguous()
    bits = 16 if w <= 16 else 32
    v = torch.where(v >= (1 << (bits - 1)), v - (1 << bits), v)
    return v.to(torch.int16 if bits == 16 else torch.int32).contiguous()


def make_request_data(torch, rng):
    n = int(math.exp(rng.uniform(math.log(MIN_ROWS), math.log(MAX_ROWS))))
    ncols = int(rng.integers(2, 7))
    while True:
        widths = [int(x) for x in rng.integers(1, 65, size=ncols)]
        if sum(widths) <= 192:
            break
    zipf = bool(rng.integers(0, 2))
    cols, card = [], []
    for w in widths:
        v = _zipf_codes(torch, rng, n, w) if zipf else _uniform_codes(torch, rng, n, w)
        cols.append(_store(torch, v, w))
        card.append(min(n, 1 << min(w, 20)) if zipf else min(n, 1 << min(w, 62)))
    return dict(n=n, widths=widths, cols=cols, card=card, zipf=zipf)


def make_trace(rng, rate, duration, pool_size):
    t, trace = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        trace.append((t, int(rng.integers(0, pool_size))))
    return trace


def warm(torch, srv, pool, rounds=2):
    """Every slot's workspace grown to what the pool needs before timing: the
    whole pool submitted at once, so that the slots share out its large
    requests (a workspace that grows in the middle of a trace would put its
    cudaMalloc, a device-wide synchronisation, on some request's latency)."""
    for _ in range(rounds):
        keep = []
        for d in pool:
            o = torch.empty(d["n"], dtype=torch.int32, device="cuda")
            keep.append((srv.submit(d["cols"], d["widths"], o, cardinality=d["card"]), o))
        for tk, _ in keep:
            srv.wait(tk)


def run_served(torch, srv, pool, trace, slots):
    """The trace through the server.  Outputs come from a ring of buffers
    allocated before timing (a buffer is reused only after its request was
    waited for), so no allocation sits inside the timed loop."""
    lat, rows, batched = [], 0, 0
    depth = 4 * slots
    maxn = max(d["n"] for d in pool)
    ring = [(torch.empty(maxn, dtype=torch.int32, device="cuda"), torch.empty(maxn, dtype=torch.int32, device="cuda"))
            for _ in range(depth + 2)]
    torch.cuda.synchronize()
    pending = []
    t0 = time.perf_counter()
    for i, (arrival, k) in enumerate(trace):
        now = time.perf_counter() - t0
        if arrival > now:
            time.sleep(arrival - now)
        d = pool[k]
        o, g = ring[i % len(ring)]
        pending.append((srv.submit(d["cols"], d["widths"], o[:d["n"]], g[:d["n"]], cardinality=d["card"]), d["n"]))
        # reap what finished, keeping the buffers in use bounded
        while len(pending) > depth:
            tk, n = pending.pop(0)
            r = srv.wait(tk)
            lat.append(r["total_ms"])
            rows += n
            batched += r["batched_with"] > 1
    for tk, n in pending:
        r = srv.wait(tk)
        lat.append(r["total_ms"])
        rows += n
        batched += r["batched_with"] > 1
    wall = time.perf_counter() - t0
    return lat, rows, wall, batched


def run_serial_plain(torch, ctx, pool, trace):
    """One request at a time, one full-array sort per original column."""
    def plain(d):
        o = torch.empty(d["n"], dtype=torch.int32, device="cuda")
        g = torch.empty(d["n"], dtype=torch.int32, device="cuda")
        g2 = torch.empty_like(g)
        ig = None
        for c, w in zip(d["cols"], d["widths"]):
            out = g if ig is not g else g2
            ctx.sort_round_plain(c, w, o, in_group=ig, out_group=out)
            ig = out

    service = {}
    for _, k in trace:
        if k not in service:
            plain(pool[k])   # warm
            t = time.perf_counter()
            plain(pool[k])
            service[k] = time.perf_counter() - t
    clock, lat, rows = 0.0, [], 0
    for arrival, k in trace:
        start = max(clock, arrival)
        clock = start + service[k]
        lat.append((clock - arrival) * 1e3)
        rows += pool[k]["n"]
    return lat, rows, clock


def benchmark(rate=200.0, duration=5.0, pool_size=32, slots=4, budget=150 << 30, batch_rows_max=1 << 20,
              seed=0xF17C0005):
    import torch
    rng = np.random.default_rng(seed)
    pool = [make_request_data(torch, rng) for _ in range(pool_size)]
    trace = make_trace(rng, rate, duration, pool_size)
    with capi.Server(0, hbm_budget_bytes=budget, slots=slots, batch_rows_max=batch_rows_max) as srv:
        warm(torch, srv, pool)
        torch.cuda.synchronize()
        lat, rows, wall, batched = run_served(torch, srv, pool, trace, slots)
    with capi.Context(0) as ctx:
        plat, prows, pwall = run_serial_plain(torch, ctx, pool, trace)
    return {
        "requests": len(trace), "rate_req_s": rate, "duration_s": duration, "slots": slots,
        "hbm_budget_gb": budget / 2**30, "batch_rows_max": batch_rows_max,
        "mean_rows_per_request": round(rows / max(1, len(lat)), 1),
        "served": {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                   "rows_per_s_M": round(rows / wall / 1e6, 1), "batched_requests": batched},
        "serial_plain": {"p50_ms": round(float(np.percentile(plat, 50)), 3),
                         "p99_ms": round(float(np.percentile(plat, 99)), 3),
                         "rows_per_s_M": round(prows / pwall / 1e6, 1)},
    }
