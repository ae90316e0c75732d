#!/usr/bin/env python
"""Benchmark of the B200 multi-column sort path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fmcs|reference]

Workload (one step): the massaged single-round plan [50] over 16,777,216 rows
of 17-bit codes (8,192 distinct values, uint32) and 33-bit codes (uint64):
stitch both columns into one 64-bit bank, sort (bank, oid) stably, emit the
group ids -- StitchComposer::run_single_plan with split {50}.  Inputs are
seeded synthetic data with the shapes of the reference's 17B33 experiment.

value:  M rows/s with the columns resident in HBM (device pointers through
        the C ABI), N GPUs = N independent replicas (weak scaling).
e2e:    the same call with pinned HOST buffers: the host->device copy of the
        columns and the device->host copy of order + group ids are inside the
        timed region.
roofline: the dominant kernel's algorithmic bytes per launch / its CUDA-event
        launch time, timed inside the library on the stream it runs on.
cpu_baseline: the reference's own composer (oracle/_ref, compiled from the
        reference sources) on the same workload, 1 host thread (its only live
        sort path is single-threaded).

--impl reference times that CPU implementation alone (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("M rows/s & HBM GB/s vs peak: batched/massaged vs plain GPU sort; "
          "p50/p99 latency")
N_ROWS = 16_777_216
SPLIT = [50]
PLAIN_SPLIT = [17, 33]
WORKLOAD = "17B33 massaged single-round plan [50], 16,777,216 rows"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------------
# byte model (algorithmic bytes per row): stitch = sources + bank;
# sort pass = 2 * (bank + oid); histogram = bank; boundary = bank + 4 (round 0)
# or bank + 8 (later rounds); gather (rounds > 0) = 4 + 2 * bank.
# --------------------------------------------------------------------------
def bank_bytes(bits: int) -> int:
    """Bank width of a sort-path split entry (src/stitch_composer.cpp:622-650)."""
    return 2 if bits <= 16 else (4 if bits <= 32 else 8)


def plan_model_bytes_per_row(col_bytes, bw, split):
    per_row = 0.0
    # stitch counted unless the bank is exactly one column at its own width
    bit = 0
    starts = np.cumsum([0] + list(bw))
    for r, w in enumerate(split):
        B = bank_bytes(w)
        lo, hi = bit, bit + w
        src = [c for c in range(len(bw)) if starts[c] < hi and starts[c + 1] > lo]
        exact = len(src) == 1 and starts[src[0]] == lo and starts[src[0] + 1] == hi and col_bytes[src[0]] == B
        if not exact:
            per_row += sum(col_bytes[c] for c in src) + B
        if r > 0:
            per_row += 4 + 2 * B
        per_row += -(-w // 8) * 2 * (B + 4) + B
        per_row += B + (4 if r == 0 else 8)
        bit = hi
    return per_row


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="fmcs_clocks_", suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], [], set()
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for name, flag in zip(self.NAMES, parts[5:9]):
                    if flag.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def visible_gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


# --------------------------------------------------------------------------
# distributed plumbing (replicas only: no collective on the data path)
# --------------------------------------------------------------------------
def dist_setup(n_gpus: int):
    """One process per GPU (torchrun env); NCCL when CUDA is present, gloo
    otherwise (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def dist_max(x: float, world: int) -> float:
    """Max over ranks (the slowest replica's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_done(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# CPU baseline: the reference's own composer (or the oracle port)
# --------------------------------------------------------------------------
def cpu_baseline(cols, bw, split, runs: int):
    from oracle import oracle as O
    n = cols[0].shape[0]
    if O.ref_available():
        secs = []
        for _ in range(runs):
            _, _, s = O.ref_run_plan_sort(cols, bw, split, final_groups=False)
            secs.append(s)
        kind = "reference"
    else:
        secs = []
        for _ in range(runs):
            t = time.perf_counter()
            O.run_plan_sort(cols, bw, split)
            secs.append(time.perf_counter() - t)
        kind = "port"
    mean = sum(secs) / len(secs)
    return {"value": n / mean / 1e6, "unit": "M rows/s", "cores": 1, "kind": kind,
            "sample": f"{runs} runs of the full {n:,}-row plan {split} (stitch + sort rounds), "
                      f"mean {mean:.3f} s per run, 1 thread",
            "seconds": secs}


# Peak host memory of one reference job on the workload (columns, the
# harness's copies, bank, order and group vectors, generation temporaries),
# with margin.
REF_JOB_BYTES = 3 << 30
REF_MAX_JOBS = 64
REF_TIME_LIMIT_S = 150.0
REF_WAIT_S = 600.0    # a job that has not reached the next barrier by then has failed


def _read_int(path):
    try:
        with open(path) as f:
            return int(f.read().split()[0])
    except (OSError, ValueError, IndexError):
        return None


def host_budget():
    """(cores, bytes) this process may use: the CPUs of its affinity mask and
    cgroup quota, and the memory available on the host and under its cgroup
    limit."""
    cores = len(os.sched_getaffinity(0))
    try:
        with open("/sys/fs/cgroup/cpu.max") as f:
            q, per = f.read().split()[:2]
        if q != "max":
            cores = min(cores, max(1, int(q) // int(per)))
    except (OSError, ValueError):
        q1 = _read_int("/sys/fs/cgroup/cpu/cpu.cfs_quota_us")
        p1 = _read_int("/sys/fs/cgroup/cpu/cpu.cfs_period_us")
        if q1 and p1 and q1 > 0:
            cores = min(cores, max(1, q1 // p1))
    import psutil
    mem = psutil.virtual_memory().available
    for lim, cur in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        l, c = _read_int(lim), _read_int(cur)
        if l and l < (1 << 60):
            mem = min(mem, l - (c or 0))
    return cores, max(0, mem)


def _ref_job(steps, warmup, barrier, out):
    """One reference job (a spawned process): the workload's columns, then
    `warmup` + `steps` full plans through the reference composer (or the
    oracle port), stopping early after REF_TIME_LIMIT_S of timed runs."""
    sys.path.insert(0, ROOT)
    from fastmulticolsort_b200 import workloads as W
    from oracle import oracle as O
    cols, bw = W.cols_17b33(N_ROWS)
    ref = O.ref_available()

    def one():
        if ref:
            return O.ref_run_plan_sort(cols, bw, SPLIT, final_groups=False)[2]
        t = time.perf_counter()
        O.run_plan_sort(cols, bw, SPLIT)
        return time.perf_counter() - t

    one()   # page the buffers in before the jobs start together
    barrier.wait(timeout=REF_WAIT_S)
    for _ in range(warmup - 1):
        one()
    barrier.wait(timeout=REF_WAIT_S)
    t0 = time.perf_counter()
    secs = []
    while len(secs) < steps and time.perf_counter() - t0 < REF_TIME_LIMIT_S:
        secs.append(one())
    out.put(secs)


def run_reference(args):
    """The reference's own composer on the host cores: its sort path is one
    thread per job, so the host runs one job per usable core (as many as the
    memory holds, at most REF_MAX_JOBS), all on the same workload at once;
    the value is the rows all jobs sorted per second of the timed phase."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    cores, mem = host_budget()
    jobs = max(1, min(cores, REF_MAX_JOBS, mem // REF_JOB_BYTES))
    if os.environ.get("FMCS_REF_JOBS"):   # fewer jobs (tests); never more than the budget
        jobs = max(1, min(jobs, int(os.environ["FMCS_REF_JOBS"])))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(jobs + 1)
    out = ctx.Queue()
    procs = [ctx.Process(target=_ref_job, args=(args.steps, args.warmup, barrier, out)) for _ in range(jobs)]
    for pr in procs:
        pr.start()
    try:
        barrier.wait(timeout=REF_WAIT_S)   # every job has its columns and one run done
        barrier.wait(timeout=REF_WAIT_S)   # warm-up done: the timed phase starts
        t0 = time.perf_counter()
        per = [out.get(timeout=REF_TIME_LIMIT_S + REF_WAIT_S) for _ in procs]
        wall = time.perf_counter() - t0
    except Exception as e:   # a job died: report it instead of waiting for good
        for pr in procs:
            if pr.is_alive():
                pr.terminate()
        print(json.dumps({"impl": "reference", "unavailable": f"a reference job failed: {type(e).__name__}"}),
              flush=True)
        return 0
    for pr in procs:
        pr.join()
    runs = sum(len(x) for x in per)
    value = runs * N_ROWS / wall / 1e6
    mean = statistics.mean(v for x in per for v in x)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "M rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / max(1, min(len(x) for x in per)) * 1e3,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded PRNG)",
        "config": {"workload": WORKLOAD, "rows": N_ROWS, "plan": SPLIT},
        "cpu_baseline": {"value": value, "unit": "M rows/s", "cores": jobs, "kind": kind,
                         "sample": f"{jobs} concurrent jobs (one per usable core: {cores} cores, "
                                   f"{mem / 2**30:.0f} GiB available), each {min(len(x) for x in per)}-"
                                   f"{max(len(x) for x in per)} full {N_ROWS:,}-row plans {SPLIT} through the "
                                   f"{'reference composer (oracle/_ref)' if kind == 'reference' else 'oracle port'}"
                                   f" (one thread each: the reference's only live sort path); {wall:.1f} s timed, "
                                   f"{mean:.3f} s per plan on average"},
        "e2e": {"value": value, "unit": "M rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
def profiled_traffic(kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary profiles/<kernel>_17b33_plan50.md (its line
    'traffic_bytes_per_launch: N'), or None."""
    import re
    path = os.path.join(ROOT, "profiles", f"{kernel}_17b33_plan50.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        m = re.search(r"^traffic_bytes_per_launch:\s*([0-9.eE+]+)", f.read(), re.M)
    return float(m.group(1)) if m else None


def time_steps(ctx, stream, fn, steps):
    import torch
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for k in range(steps):
        fn()
        evs[k + 1].record(stream)
    torch.cuda.synchronize()
    per = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    total = evs[0].elapsed_time(evs[-1])
    return total, per


def zipf_segmented(ctx, stream, n: int, reps: int):
    """Zipf-skewed segmented workload: col0 20-bit codes drawn Zipf(1.0) over 2^20
    values, col1 uniform 24-bit, col2 uniform 40-bit.  Plain comparator: one
    full-array LSD sort per column (fmcs_sort_round_plain, no segments, no
    binning); segmented: the same three rounds through the size-binned engine;
    massaged: the cost model's plan through fmcs_run_plan."""
    import torch
    from fastmulticolsort_b200 import capi
    from fastmulticolsort_b200 import workloads as W
    cols, bw = W.cols_zipf(n)
    dcols = [torch.from_numpy(c.view(np.int32 if c.dtype == np.uint32 else np.int64)).cuda() for c in cols]
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    group = torch.empty(n, dtype=torch.int32, device="cuda")
    g2 = torch.empty_like(group)
    sizes = np.bincount(cols[0].astype(np.int64), minlength=1 << 20)
    # col0 is skewed: the model's equal-group assumption takes its effective
    # cardinality (n^2 / sum of squared value counts), not its distinct count
    card = [capi.effective_cardinality(sizes), 1 << 24, min(n, 1 << 40)]
    plan, _, est = capi.optimize_plan(bw, card, [4, 4, 8], n)

    def plain():
        ctx.sort_round_plain(dcols[0], 20, order, out_group=group)
        ctx.sort_round_plain(dcols[1], 24, order, in_group=group, out_group=g2)
        ctx.sort_round_plain(dcols[2], 40, order, in_group=g2, out_group=group)

    def segmented():
        ctx.run_plan(dcols, bw, [20, 24, 40], order, group)

    def massaged():
        ctx.run_plan(dcols, bw, plan, order, group)

    out = {"rows": n, "columns": "20-bit Zipf(1.0) over 2^20 codes (u32), 24-bit (u32), 40-bit (u64)",
           "largest_group": int(sizes.max()), "groups_col0": int((sizes > 0).sum()),
           "effective_cardinality_col0": card[0], "plan_chosen": plan, "plan_est_ms": round(est, 3)}
    results = {}
    for name, fn in (("plain_ms", plain), ("segmented_ms", segmented), ("massaged_ms", massaged)):
        fn()
        total, per = time_steps(ctx, stream, fn, reps)
        out[name] = round(total / reps, 3)
        torch.cuda.synchronize()
        results[name] = (order.clone(), group.clone())   # every variant's last round writes `group`
    # the three variants must agree exactly, and the result must be a sorted,
    # canonically tie-ordered, densely grouped permutation
    from fastmulticolsort_b200 import batch_bench as BB
    same = all(torch.equal(results["plain_ms"][i], results[k][i])
               for k in ("segmented_ms", "massaged_ms") for i in (0, 1))
    props = BB.sorted_properties(torch, dcols, *results["segmented_ms"])
    out["check"] = {"variants_equal": bool(same), "properties": props,
                    "digest_order_group": BB._digest(torch, *results["segmented_ms"])}
    out["checked"] = bool(same and all(props.values()))
    del results
    best = min(out["segmented_ms"], out["massaged_ms"])
    out["speedup_vs_plain"] = round(out["plain_ms"] / best, 3)
    out["value_mrows_s"] = round(n / (best / 1e3) / 1e6, 1)
    return out


def run_fmcs(args):
    import torch
    from fastmulticolsort_b200 import capi
    from fastmulticolsort_b200 import workloads as W

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    cols, bw = W.cols_17b33(N_ROWS)
    n = N_ROWS
    col_bytes = [c.dtype.itemsize for c in cols]
    dcols = [torch.from_numpy(c.view(np.int32 if c.dtype == np.uint32 else np.int64)).cuda() for c in cols]
    dorder = torch.empty(n, dtype=torch.int32, device="cuda")
    dgroup = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx = capi.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        ctx.run_plan(dcols, bw, SPLIT, dorder, dgroup)

    def plain_step():
        ctx.run_plan(dcols, bw, PLAIN_SPLIT, dorder, dgroup)

    graph = ctx.plan_graph(dcols, bw, SPLIT, dorder, dgroup)
    gstream = torch.cuda.ExternalStream(graph.stream)

    def graph_step():
        graph.launch()

    clocks = ClockSampler(visible_gpu_index(local))
    clocks.start()
    t_load = time.perf_counter()
    for _ in range(args.warmup):
        graph_step()
        step()
    # keep the GPU busy for at least ~1 s before the timed region so that the
    # clock samples describe the loaded state
    while not args.only_steps and time.perf_counter() - t_load < 1.0:
        graph_step()
    dist_barrier(world)
    torch.cuda.synchronize()
    # timed region: K replays of the captured plan (device-resident columns)
    total_ms, per_ms = time_steps(ctx, gstream, graph_step, args.steps)
    torch.cuda.synchronize()
    dist_barrier(world)
    clk = clocks.stop()
    total_ms = dist_max(total_ms, world)
    ms_per_step = total_ms / args.steps
    value = world * n / (ms_per_step / 1e3) / 1e6
    # the timed replays' result: a sorted, canonically tie-ordered, densely
    # grouped permutation of the rows (size-independent checks on the device)
    from fastmulticolsort_b200 import batch_bench as BB
    head_props = BB.sorted_properties(torch, dcols, dorder, dgroup)
    head_check = {"properties": head_props, "digest_order_group": BB._digest(torch, dorder, dgroup)}
    # the same K steps as eager C-ABI calls, with the library's CUDA events
    # around every kernel: the per-kernel split and the roofline.  An eager
    # step launches the same kernels as a replay (the replay's level loop runs
    # as many levels as the eager host loop), so its launch count per step is
    # the replay's.
    ctx.profile(True)
    lc0 = ctx.launch_count()
    eager_total, _ = time_steps(ctx, stream, step, args.steps)
    launches = (ctx.launch_count() - lc0) // max(1, args.steps) * args.steps
    prof = {k: v for k, v in ctx.profile_report().items() if not k.startswith("_")}
    ctx.profile(False)
    eager_ms = dist_max(eager_total / args.steps, world)
    if args.only_steps:
        graph.close()
        ctx.close()
        dist_done(world)
        if rank == 0:
            print(json.dumps({"only_steps": True, "value": value, "ms_per_step": ms_per_step,
                              "eager_ms_per_step": eager_ms, "kernels": prof}), flush=True)
        return 0

    # plain one-sort-per-column comparator on the same data
    for _ in range(3):
        plain_step()
    plain_total, _ = time_steps(ctx, stream, plain_step, max(3, args.steps // 2))
    plain_ms = dist_max(plain_total / max(3, args.steps // 2), world)

    # every bit-borrowing split [17-k, 33+k], k = 0..17 (k = 17 is [50]), the
    # exhaustive sweep the cost model's choice is checked against
    sweep = {}
    for k in range(0, 18):
        sp = W.split_for_k(k)
        fn = (lambda sp=sp: ctx.run_plan(dcols, bw, sp, dorder, dgroup))
        fn()
        tot, _ = time_steps(ctx, stream, fn, 5)
        sweep[str(sp)] = round(dist_max(tot / 5, world), 4)
    card = [8192, n]
    opt_split, _, opt_est = capi.optimize_plan(bw, card, col_bytes, n)
    best = min(sweep, key=sweep.get)
    split_sweep = {"ms_per_plan": sweep, "fastest": best, "cost_model_choice": opt_split,
                   "cost_model_est_ms": round(opt_est, 4),
                   "choice_ms": sweep.get(str(opt_split)),
                   "choice_vs_fastest": round(sweep.get(str(opt_split), float("nan")) / sweep[best], 3)}

    # end to end: pinned host buffers, copies inside the timed region
    hcols = []
    for c in cols:
        t = torch.empty(c.shape[0], dtype=torch.int32 if c.dtype == np.uint32 else torch.int64, pin_memory=True)
        t.numpy()[:] = c.view(t.numpy().dtype)
        hcols.append(t.numpy().view(c.dtype))
    horder = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    hgroup = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)

    def e2e_step():
        ctx.run_plan(hcols, bw, SPLIT, horder, hgroup)

    for _ in range(2):
        e2e_step()
    e2e_steps = max(3, min(args.steps, 20))
    e2e_total, _ = time_steps(ctx, stream, e2e_step, e2e_steps)
    e2e_ms = dist_max(e2e_total / e2e_steps, world)
    e2e_value = world * n / (e2e_ms / 1e3) / 1e6

    # the same steps through the serving loop (fmcs_server): two slots, each a
    # stream of its own, so one step's host->device copies run beside another
    # step's kernels and device->host copies; each step still copies its
    # columns in and its order and group ids out inside the timed region
    outs = [(torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32),
             torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)) for _ in range(2)]
    with capi.Server(local, hbm_budget_bytes=150 << 30, slots=2, batch_rows_max=0) as srv:
        # warm both slots (submitted together, so that each runs one): a slot
        # whose workspace grew inside the timed steps would put a cudaMalloc,
        # a device-wide synchronisation, between the other slot's copies
        for _ in range(2):
            warm = [srv.submit(hcols, bw, outs[k][0], outs[k][1], split=SPLIT) for k in range(2)]
            for t in warm:
                srv.wait(t)
        dist_barrier(world)
        t0 = time.perf_counter()
        tickets = []
        for k in range(e2e_steps):
            if k >= 2:
                srv.wait(tickets[k - 2])   # frees the output buffers this step reuses
            tickets.append(srv.submit(hcols, bw, outs[k % 2][0], outs[k % 2][1], split=SPLIT))
        for t in tickets[-2:]:
            srv.wait(t)
        pipe_ms = dist_max((time.perf_counter() - t0) * 1e3 / e2e_steps, world)
    e2e_pipe_value = world * n / (pipe_ms / 1e3) / 1e6

    # roofline of the dominant kernel that reports its rows
    hbm_peak, peak_kind = peaks()
    dom, dom_ms = None, 0.0
    for name, rec in prof.items():
        if rec.get("bytes", 0) > 0 and rec["ms"] > dom_ms:
            dom, dom_ms = name, rec["ms"]
    roofline = None
    if dom:
        rec = prof[dom]
        bytes_total = rec["bytes"]   # the library's algorithmic bytes of the launches
        achieved = bytes_total / (rec["ms"] / 1e3) / 1e9
        traffic = profiled_traffic(dom)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm_peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                    "traffic": traffic,
                    "bytes_per_launch": bytes_total / rec["launches"],
                    "launch_ms": rec["ms"] / rec["launches"], "launches": rec["launches"]}
    model_bpr = plan_model_bytes_per_row(col_bytes, bw, SPLIT)
    plan_gbs = model_bpr * n / (ms_per_step / 1e3) / 1e9
    total_kernel_ms = sum(r["ms"] for r in prof.values())

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "M rows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded PRNG; 17-bit codes from 8,192 distinct values + uniform 33-bit codes)",
        "config": {"workload": WORKLOAD, "rows": n, "plan": SPLIT, "columns": "u32 (17 bits) + u64 (33 bits)",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (192 MB of columns)",
                   "launch": "CUDA-graph replay of the plan (fmcs_graph_launch); eager C-ABI calls in eager_ms"},
        "eager_ms_per_step": round(eager_ms, 4),
        "latency_ms": {"p50": round(float(np.percentile(per_ms, 50)), 4),
                       "p99": round(float(np.percentile(per_ms, 99)), 4)},
        "plan_hbm": {"model_bytes_per_row": model_bpr, "achieved_gbs": round(plan_gbs, 1),
                     "frac_of_peak": round(plan_gbs / hbm_peak, 4)},
        "plain_gpu": {"plan": PLAIN_SPLIT, "value": round(world * n / (plain_ms / 1e3) / 1e6, 2),
                      "ms_per_step": round(plain_ms, 4),
                      # both eager: the same calls, only the plan differs
                      "speedup_of_massaged": round(plain_ms / eager_ms, 3)},
        "split_sweep": split_sweep,
        "roofline": roofline,
        "kernels": {k: {"launches_per_step": v["launches"] / args.steps, "ms_per_step": round(v["ms"] / args.steps, 4)}
                    for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])},
        "kernel_ms_per_step": round(total_kernel_ms / args.steps, 4),
        "e2e": {"value": round(e2e_value, 2), "unit": "M rows/s", "ms_per_step": round(e2e_ms, 4),
                "h2d_bytes_per_step": int(sum(c.nbytes for c in cols)), "d2h_bytes_per_step": int(8 * n)},
        "e2e_pipelined": {"value": round(e2e_pipe_value, 2), "unit": "M rows/s", "ms_per_step": round(pipe_ms, 4),
                          "how": "fmcs_server, 2 slots: consecutive steps' copies and kernels overlap",
                          "h2d_bytes_per_step": int(sum(c.nbytes for c in cols)), "d2h_bytes_per_step": int(8 * n)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "check": head_check,
        "checked": all(head_props.values()),
    }
    if not args.no_zipf:
        line["zipf_segmented"] = zipf_segmented(ctx, stream, args.zipf_rows, max(3, min(args.steps, 10)))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cols, bw, SPLIT, args.cpu_runs)
        line["cpu_baseline"].pop("seconds", None)
    graph.close()
    ctx.close()
    dist_done(world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    """Serving-loop workload: one JSON line of its own."""
    from fastmulticolsort_b200 import serving
    res = serving.benchmark(rate=args.rate, duration=args.duration)
    line = {"metric": METRIC, "workload": "serving", "value": res["served"]["rows_per_s_M"], "unit": "M rows/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic (seeded; generated on the device)",
            "latency_ms": {"p50": res["served"]["p50_ms"], "p99": res["served"]["p99_ms"]},
            "config": {"workload": "Poisson 200 req/s, rows log-uniform [65536, 67108864], 2-6 columns of 1-64 "
                                   "bits, uniform or Zipf(0.8) codes, columns resident, 150 GB admission budget"},
            **res}
    print(json.dumps(line), flush=True)
    return 0


def run_batch_workloads(args):
    """Many independent instances and the wide table: one JSON line of their own."""
    from fastmulticolsort_b200 import batch_bench
    res = batch_bench.benchmark(reps=max(1, min(args.steps, 5)), with_instances=not args.no_instances,
                                wide_rows=args.wide_rows)
    inst = res.get("instances")
    wd = res["wide"]
    line = {"metric": METRIC, "workload": "batch",
            "value": inst["batched_mrows_s"] if inst else wd["order_by_mrows_s"], "unit": "M rows/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic (seeded; generated on the device)",
            "config": {"workload": (f"{inst['instances']} instances, {inst['rows']:,} rows in all (8/24/40-bit "
                                    "columns), one fmcs_run_batch call; plus " if inst else "")
                       + f"a {args.wide_rows:,}-row 6-column wide table"},
            **res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fmcs", choices=["fmcs", "reference"])
    ap.add_argument("--cpu-runs", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-zipf", action="store_true", help="skip the Zipf segmented comparison")
    ap.add_argument("--zipf-rows", type=int, default=67_108_864)
    ap.add_argument("--workload", default="massaged", choices=["massaged", "serving", "batch"])
    ap.add_argument("--no-instances", action="store_true", help="batch workload: the wide table only")
    ap.add_argument("--wide-rows", type=int, default=60_000_000, help="batch workload: rows of the wide table")
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--only-steps", action="store_true",
                    help="warm-up and timed steps only (no comparators, e2e or CPU baseline): "
                         "the command the ncu captures profile")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "batch":
        return run_batch_workloads(args)
    return run_fmcs(args)


if __name__ == "__main__":
    sys.exit(main())
