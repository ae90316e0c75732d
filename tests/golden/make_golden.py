"""Generate tests/golden/golden.npz from the REFERENCE implementation.

Runs FastMultiColSort's own composer (oracle/_ref/libfmcs_ref.so, compiled
from the reference sources by oracle/Makefile) on small seeded inputs and
stores inputs + canonicalised outputs (ties sorted to ascending oid inside
each final group, the reference's sort being unstable).  The committed
fixture pins the oracle and the CUDA path without the reference present.

    python tests/golden/make_golden.py

Hash cases keep every parent range <= the reference's hash block size or a
multiple of it, where src/hashing.h:345 (remainder-block defect) is harmless.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fastmulticolsort_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def cases():
    c = []
    cols, bw = W.cols_17b33(8192, seed_index=101)
    for split in ([17, 33], [50], [6, 44], [9, 41], [1, 49], [16, 34], [17 - 8, 33 + 8]):
        c.append(("17b33", cols, bw, split, "sort"))
    cols, bw = W.cols_zipf(12000, seed_index=103, ranks_bits=20)
    for split in ([20, 24, 40], [20, 64], [44, 40], [12, 36, 36]):
        c.append(("zipf", cols, bw, split, "sort"))
    cols, bw = W.cols_uniform(10000, [8, 24, 40], seed_index=104, distinct=[16, 0, 0])
    for split in ([8, 24, 40], [32, 40], [8, 64], [16, 56]):
        c.append(("u8_24_40", cols, bw, split, "sort"))
    cols, bw = W.cols_uniform(16384, [2, 1, 12, 12, 32, 7], seed_index=105,
                              distinct=[3, 2, 2526, 2526, 0, 100])
    for split in ([2, 1, 12, 12, 32, 7], [27, 39], [15, 51], [3, 24, 39]):
        c.append(("wide6", cols, bw, split, "sort"))
    # (a u8 hash bank built from two slices is outside the parity domain: the
    # reference's SpecialiedColumn<uint8_t>::ShiftLeftBatch is empty,
    # src/column.h:105-110, so it ORs the slices unshifted)
    for split in ([27, 39], [16, 50], [2, 25, 39]):
        c.append(("wide6", cols, bw, split, "hash"))
    cols, bw = W.cols_uniform(16384, [8, 12, 7], seed_index=106, distinct=[16, 100, 0])
    for split in ([8, 12, 7], [27], [20, 7], [8, 19]):
        c.append(("u8_12_7", cols, bw, split, "hash"))
    # the 9-tuple fixture of the reference's tests/subgroup_test.cpp:98-145
    c1 = np.array([100, 200, 200, 200, 100, 100, 300, 100, 100], np.uint32)
    c2 = np.array([1000, 2000, 2000, 1000, 2000, 1000, 3000, 4000, 4000], np.uint32)
    for split in ([32, 32], [64]):
        c.append(("subgroup9", [c1, c2], [32, 32], split, "hash"))
        c.append(("subgroup9", [c1, c2], [32, 32], split, "sort"))
    # tiny and ragged sizes
    for n in (1, 2, 3, 31, 33, 127, 129, 1000):
        cols, bw = W.cols_17b33(n, seed_index=200 + n)
        c.append((f"17b33_n{n}", cols, bw, [50], "sort"))
        c.append((f"17b33_n{n}", cols, bw, [17, 33], "sort"))
    return c


SMALL = 1000


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def main():
    O.build()
    arrays = {}
    meta = []
    for k, (name, cols, bw, split, path) in enumerate(cases()):
        if path == "sort":
            order, group, _ = O.ref_run_plan_sort(cols, bw, split, final_groups=True)
            order = O.canonicalize(order, group)
        else:
            order, group, _ = O.ref_run_plan_hash(cols, bw, split)
        for ci, col in enumerate(cols):
            key = f"in_{name}_col{ci}"
            if key not in arrays:
                arrays[key] = col
        entry = {"case": k, "name": name, "bw": bw, "split": split, "path": path,
                 "ncols": len(cols), "n": int(cols[0].shape[0]),
                 "ngroups": int(group.max()) + 1 if group.size else 0,
                 "order_sha256": digest(order), "group_sha256": digest(group)}
        if order.shape[0] <= SMALL:
            arrays[f"c{k}_order"] = order
            arrays[f"c{k}_group"] = group
        meta.append(entry)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {len(meta)} cases to {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
