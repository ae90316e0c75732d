"""The autotuner's file round-trips into both of its readers: the cost model
(GpuCostTables::Load, through fmcs_optimize_plan's estimate; no GPU needed)
and a context's knobs (fmcs_get_tuning, on a GPU), and a sort with the tuned
knobs still matches the oracle exactly.  The reference's counterpart is the
hand-calibrated tables of src/params.h:200-2283."""
import json
import os
import subprocess
import sys

import pytest

from fastmulticolsort_b200 import autotune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(code: str, tuning: str) -> dict:
    env = dict(os.environ, FMCS_TUNING=tuning, PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True,
                         timeout=300)
    return json.loads(out.stdout.strip().splitlines()[-1])


def _scaled(path: str, factor: float, knobs: dict) -> None:
    base = json.load(open(autotune.DEFAULT_OUT))
    tables = {"stitch_per_byte": base["stitch_per_byte"] * factor,
              "gather": [x * factor for x in base["gather"]],
              "boundary": [x * factor for x in base["boundary"]],
              "msd_level": [x * factor for x in base["msd_level"]],
              "local": [[x * factor for x in row] for row in base["local"]],
              "round_fixed_ms": base["round_fixed_ms"] * factor}
    autotune.write_tuning(path, knobs, tables, "test")


ESTIMATE = """
import json
from fastmulticolsort_b200 import capi
out = {}
for name, bw, card, cb, n in (("17b33", [17, 33], [8192, 1 << 24], [4, 8], 1 << 24),
                              ("wide", [2, 1, 12, 12, 32, 7], [3, 2, 2526, 2526, 60_000_000, 100],
                               [2, 2, 2, 2, 4, 2], 60_000_000)):
    split, order, est = capi.optimize_plan(bw, card, cb, n)
    out[name] = [split, order, est]
print(json.dumps(out))
"""


def test_cost_tables_round_trip(tmp_path):
    """Every table doubled: the optimizer's estimates double and its choices
    stay the same (the relative costs did not change)."""
    knobs = {"rank_mode": 2, "local_max": 8192, "msd_items": 16}
    one, two = str(tmp_path / "x1.json"), str(tmp_path / "x2.json")
    _scaled(one, 1.0, knobs)
    _scaled(two, 2.0, knobs)
    a = _run(ESTIMATE, one)
    b = _run(ESTIMATE, two)
    for k in a:
        assert a[k][0] == b[k][0] and a[k][1] == b[k][1]
        assert b[k][2] == pytest.approx(2.0 * a[k][2], rel=1e-9)


KNOBS = """
import json
import numpy as np
from fastmulticolsort_b200 import capi, workloads as W
from oracle import oracle as O
with capi.Context(0) as ctx:
    got = {k: ctx.get_tuning(k) for k in ("rank_mode", "local_max", "msd_items")}
    cols, bw = W.cols_17b33(1 << 20, seed_index=77)
    n = cols[0].shape[0]
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.run_plan(cols, bw, [50], order, group)
    o, g, ng_ref = O.run_plan_sort(cols, bw, [50])
    got["exact"] = bool(ng == ng_ref and np.array_equal(order, o) and np.array_equal(group, g))
print(json.dumps(got))
"""


@pytest.mark.gpu
@pytest.mark.parametrize("knobs", [{"rank_mode": 1, "local_max": 4096, "msd_items": 8},
                                   {"rank_mode": 0, "local_max": 2048, "msd_items": 16}])
def test_context_knobs_round_trip(tmp_path, knobs):
    path = str(tmp_path / "k.json")
    _scaled(path, 1.0, knobs)
    got = _run(KNOBS, path)
    assert got.pop("exact")
    assert got == knobs
