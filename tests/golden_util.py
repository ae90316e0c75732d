"""Loader of tests/golden/golden.npz (made by tests/golden/make_golden.py from
the reference's own composer)."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def load_cases():
    z = np.load(PATH)
    meta = json.loads(bytes(z["meta"]).decode())
    out = []
    for m in meta:
        cols = [z[f"in_{m['name']}_col{ci}"] for ci in range(m["ncols"])]
        k = m["case"]
        small = f"c{k}_order" in z.files
        out.append(dict(m, cols=cols,
                        order=z[f"c{k}_order"] if small else None,
                        group=z[f"c{k}_group"] if small else None))
    return out


def case_id(c) -> str:
    return f"{c['case']}-{c['name']}-{c['path']}-{'B'.join(map(str, c['split']))}"
