"""Autotuner of the B200 sort engine.

Picks the engine's knobs -- multi-split ranking mode, the largest segment
sorted on chip (``local_max``: the warp/block tiers versus the HBM radix
levels) and the HBM radix tile (``msd_items``) -- by timing representative
workloads, then re-measures the cost model's per-bank-width tables (stitch,
gather, group-id scan, one HBM radix level, on-chip sorts by group size) with
the chosen knobs, in milliseconds per million rows.  The result is one JSON
file that both the library (knobs, at context creation) and the C++ cost model
(GpuCostTables::Load) read: ``fastmulticolsort_b200/tuning/b200.json`` next to
``libfmcs.so`` (or the file named by FMCS_TUNING).

The reference's equivalent is the hand-calibrated cycle tables of
src/params.h:200-2283 for one Haswell core.

    python -m fastmulticolsort_b200.autotune --out <file.json> [--quick]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import statistics
import time

import numpy as np

from . import capi
from . import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuning", "b200.json")
KNOBS = {"rank_mode": (0, 1, 2), "local_max": (2048, 4096, 8192), "msd_items": (8, 16)}


def _dev(a):
    import torch
    return torch.from_numpy(a.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[a.dtype.itemsize])).cuda()


def _time(fn, reps: int) -> float:
    """Median milliseconds of fn() (the C-ABI calls return when done)."""
    fn()
    ts = []
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        ts.append((time.perf_counter() - t) * 1e3)
    return statistics.median(ts)


class Workloads:
    """Device-resident inputs of the knob search."""

    def __init__(self, quick: bool):
        import torch
        n = 1 << (22 if quick else 24)
        cols, self.bw = W.cols_17b33(n, seed_index=61)
        self.cols = [_dev(c) for c in cols]
        self.n = n
        # a segmented round on skewed groups: round 1 of [20, 24, 40]
        zc, _ = W.cols_zipf(n, seed_index=62)
        z0 = _dev(zc[0])
        self.z1 = _dev(zc[1])
        self.order = torch.zeros(n, dtype=torch.int32, device="cuda")
        self.group = torch.zeros(n, dtype=torch.int32, device="cuda")
        self.zorder = torch.zeros(n, dtype=torch.int32, device="cuda")
        self.zgroup = torch.zeros(n, dtype=torch.int32, device="cuda")
        with capi.Context(0) as c:
            c.sort_round(z0, 20, self.zorder, out_group=self.zgroup)
        self.tmp_order = torch.empty_like(self.zorder)
        self.tmp_group = torch.empty_like(self.zgroup)

    def run(self, ctx) -> float:
        a = _time(lambda: ctx.run_plan(self.cols, self.bw, [50], self.order, self.group), 5)

        def seg():
            self.tmp_order.copy_(self.zorder)
            ctx.sort_round(self.z1, 24, self.tmp_order, in_group=self.zgroup, out_group=self.tmp_group)
        b = _time(seg, 5)
        return a + b


def search_knobs(ctx, wl: Workloads):
    results = []
    for values in itertools.product(*KNOBS.values()):
        knobs = dict(zip(KNOBS.keys(), values))
        for k, v in knobs.items():
            ctx.set_tuning(k, v)
        ms = wl.run(ctx)
        results.append((ms, knobs))
    results.sort(key=lambda r: r[0])
    best = results[0][1]
    for k, v in best.items():
        ctx.set_tuning(k, v)
    return best, [{"ms": round(ms, 4), **kn} for ms, kn in results]


def calibrate(ctx, quick: bool) -> dict:
    import torch
    n = 1 << (22 if quick else 24)
    mrows = n / 1e6
    rng = np.random.default_rng(7)
    out = {}
    # stitch: a u32 and a u64 source into a u64 bank (20 bytes moved per row)
    a = _dev(rng.integers(0, 1 << 17, size=n, dtype=np.uint64).astype(np.uint32))
    b = _dev(rng.integers(0, 1 << 33, size=n, dtype=np.uint64))
    bank = torch.empty(n, dtype=torch.int64, device="cuda")
    ms = _time(lambda: ctx.stitch([(a, 17, 1, 17), (b, 33, 1, 33)], bank), 7)
    out["stitch_per_byte"] = ms / mrows / 20.0
    order = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda()
    gather, boundary, msd, local = [], [], [], []
    for nb, dt in ((2, torch.int16), (4, torch.int32), (8, torch.int64)):
        bits = 8 * nb
        src = _dev(rng.integers(0, 1 << min(bits, 62), size=n, dtype=np.uint64).astype(np.dtype(f"u{nb}")))
        dst = torch.empty(n, dtype=dt, device="cuda")
        gather.append(_time(lambda: ctx.gather(src, order, dst), 7) / mrows)
        # one HBM radix level (round 0 over uniform keys, MSD kernels only) and
        # the boundary scan of the round's group ids, both timed inside the
        # round as the library runs them
        o = torch.empty(n, dtype=torch.int32, device="cuda")
        grp = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.sort_round(src, bits, o, out_group=grp)
        ctx.profile(True)
        ctx.sort_round(src, bits, o, out_group=grp)
        prof = ctx.profile_report()
        ctx.profile(False)
        boundary.append(prof["boundary_scan"]["ms"] / mrows)
        lvl_ms = sum(v["ms"] for k, v in prof.items() if k.startswith(("msd_", "tile_prefix")))
        rows = prof.get("msd_scatter", {}).get("units", 0) or n
        msd.append(lvl_ms / (rows / 1e6))
        # on-chip sorts of groups of 2^k rows
        row = [0.0]
        for k in range(1, 14):
            size = 1 << k
            ig = torch.arange(n, dtype=torch.int32, device="cuda") // size
            oo = torch.arange(n, dtype=torch.int32, device="cuda")
            gg = torch.empty(n, dtype=torch.int32, device="cuda")
            ctx.sort_round(src, bits, oo.clone(), in_group=ig, out_group=gg)
            ctx.profile(True)
            ctx.sort_round(src, bits, oo.clone(), in_group=ig, out_group=gg)
            prof = ctx.profile_report()
            ctx.profile(False)
            lm = sum(v["ms"] for kk, v in prof.items()
                     if kk.startswith(("warp_sort", "block_sort", "copy", "classify", "msd_", "tile_prefix")))
            row.append(lm / mrows)
        local.append(row)
    out["gather"] = gather
    out["boundary"] = boundary
    out["msd_level"] = msd
    out["local"] = local
    tiny = np.arange(1024, dtype=np.uint32)[::-1].copy()
    to = np.zeros(1024, np.uint32)
    out["round_fixed_ms"] = _time(lambda: ctx.sort_round(tiny, 10, to), 21)
    return out


def write_tuning(path: str, knobs: dict, tables: dict, how: str, knob_search=None) -> dict:
    """The tuning file both readers take: the library's context knobs
    (rank_mode, local_max, msd_items) and the cost model's tables
    (GpuCostTables::Load: stitch_per_byte, gather, boundary, msd_level, local,
    round_fixed_ms), in ms per million rows."""
    doc = {"device": "B200", "how": how, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           **knobs, **tables, "knob_search": knob_search or []}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
    return doc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--quick", action="store_true")
    args = ap.parse_args()
    with capi.Context(0) as ctx:
        wl = Workloads(args.quick)
        best, table = search_knobs(ctx, wl)
        tables = calibrate(ctx, args.quick)
    write_tuning(args.out, best, tables, "python -m fastmulticolsort_b200.autotune" + (" --quick" if args.quick else ""),
                 table)
    print(json.dumps({"best": best, "out": args.out}))


if __name__ == "__main__":
    main()
