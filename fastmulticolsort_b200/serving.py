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


def warm(torch, srv, pool, slots, rounds=1):
    """Every slot's workspace grown to what the pool needs before timing (a
    workspace that grows in the middle of a trace puts its cudaMalloc, a
    device-wide synchronisation, on the latency of every request in flight):
    each request of the pool, largest first, submitted `slots` times at once so
    that every slot runs it; then the whole pool at once, so that the shared
    launches of small requests are warm too."""
    for d in sorted(pool, key=lambda d: -d["n"]):
        keep = []
        for _ in range(slots):
            o = torch.empty(d["n"], dtype=torch.int32, device="cuda")
            keep.append((srv.submit(d["cols"], d["widths"], o, cardinality=d["card"]), o))
        for tk, _ in keep:
            srv.wait(tk)
    for _ in range(rounds):
        keep = []
        for d in pool:
            o = torch.empty(d["n"], dtype=torch.int32, device="cuda")
            keep.append((srv.submit(d["cols"], d["widths"], o, cardinality=d["card"]), o))
        for tk, _ in keep:
            srv.wait(tk)


def run_served(torch, srv, pool, trace, slots, keep=None):
    """The trace through the server.  Outputs come from a ring of buffers
    allocated before timing (a buffer is reused only after its request was
    waited for), so no allocation sits inside the timed loop.  Returns the
    latencies (ms, in trace order), rows, wall seconds, the number of requests
    that ran inside a shared launch, and, for the requests whose trace index
    is in `keep`, a copy of their (order, group) and their batch size."""
    lat, rows, batched = [], 0, 0
    kept = {}
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
        pending.append((srv.submit(d["cols"], d["widths"], o[:d["n"]], g[:d["n"]], cardinality=d["card"]), d["n"],
                        i, o, g))
        # reap what finished, keeping the buffers in use bounded
        while len(pending) > depth:
            tk, n, j, oo, gg = pending.pop(0)
            r = srv.wait(tk)
            lat.append(r["total_ms"])
            rows += n
            batched += r["batched_with"] > 1
            if keep is not None and j in keep:
                kept[j] = (oo[:n].clone(), gg[:n].clone(), r["batched_with"])
    for tk, n, j, oo, gg in pending:
        r = srv.wait(tk)
        lat.append(r["total_ms"])
        rows += n
        batched += r["batched_with"] > 1
        if keep is not None and j in keep:
            kept[j] = (oo[:n].clone(), gg[:n].clone(), r["batched_with"])
    wall = time.perf_counter() - t0
    if keep is not None:
        return lat, rows, wall, batched, kept
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


def burst_trace(rng, bursts, per_burst, gap_s, pool_size):
    """Bursts of `per_burst` requests arriving together every `gap_s` seconds
    (requests that co-arrive while the slots are busy: the case continuous
    batching is for)."""
    trace = []
    for b in range(bursts):
        for _ in range(per_burst):
            trace.append((b * gap_s, int(rng.integers(0, pool_size))))
    return trace


def burst_benchmark(torch, slots=4, budget=150 << 30, batch_rows_max=1 << 20, seed=0xF17C0006, bursts=40,
                    per_burst=48, gap_s=0.025, pool_size=48):
    """Small requests (65,536 to 1,048,576 rows, log-uniform) of ONE layout
    (8/24/40-bit uniform columns, the many-instances shape) in bursts, served
    with continuous batching (batch_rows_max) and without it (0); a sample of
    the requests' results from the batched run is compared with the same
    requests' results from the unbatched run."""
    rng = np.random.default_rng(seed)
    widths = [8, 24, 40]
    pool = []
    for _ in range(pool_size):
        n = int(math.exp(rng.uniform(math.log(MIN_ROWS), math.log(1 << 20))))
        cols = [_store(torch, _uniform_codes(torch, rng, n, w), w) for w in widths]
        pool.append(dict(n=n, widths=widths, cols=cols, card=[min(n, 1 << w) for w in widths], zipf=False))
    trace = burst_trace(rng, bursts, per_burst, gap_s, pool_size)
    keep = set(range(0, len(trace), max(1, len(trace) // 16)))
    out = {"requests": len(trace), "bursts": bursts, "per_burst": per_burst, "gap_ms": gap_s * 1e3,
           "rows": "log-uniform [65536, 1048576]", "columns": widths}
    results = {}
    for name, brm in (("batched", batch_rows_max), ("unbatched", 0)):
        with capi.Server(0, hbm_budget_bytes=budget, slots=slots, batch_rows_max=brm) as srv:
            warm(torch, srv, pool, slots)
            torch.cuda.synchronize()
            lat, rows, wall, nb, kept = run_served(torch, srv, pool, trace, slots, keep=keep)
        results[name] = kept
        out[name] = {"p50_ms": round(float(np.percentile(lat, 50)), 3),
                     "p99_ms": round(float(np.percentile(lat, 99)), 3),
                     "rows_per_s_M": round(rows / wall / 1e6, 1), "batched_requests": nb,
                     "batch_rows_max": brm}
    same = all(torch.equal(results["batched"][j][0], results["unbatched"][j][0])
               and torch.equal(results["batched"][j][1], results["unbatched"][j][1]) for j in keep)
    out["check"] = {"sampled": len(keep),
                    "sampled_in_shared_launch": int(sum(results["batched"][j][2] > 1 for j in keep)),
                    "batched_equals_unbatched": bool(same)}
    out["checked"] = bool(same)
    return out


def tail_of(lat, trace, pool, q=99):
    """The requests at or above the q-th latency percentile: how many, and
    their mean rows and key bits, beside the trace's mean rows (what the
    tail is made of)."""
    lat = np.asarray(lat)
    cut = np.percentile(lat, q)
    ds = [pool[trace[i][1]] for i, v in enumerate(lat) if v >= cut and i < len(trace)]
    if not ds:
        return {}
    return {"count": len(ds), "mean_rows": round(float(np.mean([d["n"] for d in ds])), 1),
            "mean_key_bits": round(float(np.mean([sum(d["widths"]) for d in ds])), 1),
            "trace_mean_rows": round(float(np.mean([pool[k]["n"] for _, k in trace])), 1)}


def benchmark(rate=200.0, duration=5.0, pool_size=32, slots=4, budget=150 << 30, batch_rows_max=1 << 20,
              seed=0xF17C0005):
    import torch
    rng = np.random.default_rng(seed)
    pool = [make_request_data(torch, rng) for _ in range(pool_size)]
    trace = make_trace(rng, rate, duration, pool_size)
    with capi.Server(0, hbm_budget_bytes=budget, slots=slots, batch_rows_max=batch_rows_max) as srv:
        warm(torch, srv, pool, slots)
        torch.cuda.synchronize()
        lat, rows, wall, batched = run_served(torch, srv, pool, trace, slots)
    with capi.Context(0) as ctx:
        plat, prows, pwall = run_serial_plain(torch, ctx, pool, trace)
    burst = burst_benchmark(torch, slots=slots, budget=budget, batch_rows_max=batch_rows_max)
    return {
        "requests": len(trace), "rate_req_s": rate, "duration_s": duration, "slots": slots,
        "hbm_budget_gb": budget / 2**30, "batch_rows_max": batch_rows_max,
        "mean_rows_per_request": round(rows / max(1, len(lat)), 1),
        "served": {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                   "rows_per_s_M": round(rows / wall / 1e6, 1), "batched_requests": batched},
        "serial_plain": {"p50_ms": round(float(np.percentile(plat, 50)), 3),
                         "p99_ms": round(float(np.percentile(plat, 99)), 3),
                         "rows_per_s_M": round(prows / pwall / 1e6, 1)},
        "p99_tail": tail_of(lat, trace, pool),
        "burst": burst,
    }
