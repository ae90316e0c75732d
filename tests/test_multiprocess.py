"""The N>1 plumbing of bench.py on CPU: one process per rank over gloo, the
max-over-ranks timing, and the reference arm's rank handling (rank 0 runs
and prints one line, the other ranks exit 0 without work)."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, w, _ = bench.dist_setup(world)
    assert (r, w) == (rank, world)
    bench.dist_barrier(w)
    m = bench.dist_max(10.0 + rank, w)
    out[rank] = m
    bench.dist_done(w)


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29517
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 11.0


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libfmcs_ref.so")),
                    reason="reference harness not built")
def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", "29518", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, FMCS_REF_JOBS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1   # rank 0 alone reports
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["cores"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_host_budget_reports_usable_cores_and_memory():
    """The reference arm sizes its job count from these: the CPUs of the
    affinity mask (capped by any cgroup quota) and the memory available."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    cores, mem = bench.host_budget()
    assert 1 <= cores <= len(os.sched_getaffinity(0))
    assert mem > 0
    assert max(1, min(cores, bench.REF_MAX_JOBS, mem // bench.REF_JOB_BYTES)) >= 1
