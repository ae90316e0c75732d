"""ctypes front end of the parity oracle: the C restatement (``_build/liboracle.so``)
and, where it was built, the reference's own composer (``_ref/libfmcs_ref.so``).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` import this module, and only as
the parity oracle or the timed CPU baseline.  The product path never does.

Every function mirrors one C entry point of ``fmcs_oracle.h`` or
``ref_harness.cpp``; those files cite the reference code they follow.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfmcs_ref.so")

_u32p = C.POINTER(C.c_uint32)


class _Slice(C.Structure):
    _fields_ = [("src", C.c_void_p), ("src_bytes", C.c_uint32), ("src_bits", C.c_uint32),
                ("start", C.c_uint32), ("end", C.c_uint32)]


class _Record(C.Structure):
    _fields_ = [("final_idx", C.c_uint32), ("start", C.c_uint32), ("end", C.c_uint32)]


_lib = None
_ref = None


def build() -> None:
    """Compile the C restatement (and the reference harness when the reference
    tree is present) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_plan_records.argtypes = [_u32p, C.c_uint32, _u32p, _u32p, C.c_uint32,
                                       C.POINTER(_Record), _u32p]
        L.orc_bank_bytes.argtypes = [C.c_uint32, C.c_int]
        L.orc_bank_bytes.restype = C.c_uint32
        L.orc_stitch.argtypes = [C.POINTER(_Slice), C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint64]
        L.orc_sort_round.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_uint64, _u32p]
        L.orc_hash_round.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_uint64, C.c_int, _u32p]
        L.orc_hash_unordered.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, _u32p]
        for f in (L.orc_run_plan_sort, L.orc_run_plan_hash):
            f.argtypes = [C.POINTER(C.c_void_p), _u32p, _u32p, C.c_uint32, _u32p, _u32p, C.c_uint32,
                          C.c_uint64, C.c_void_p, C.c_void_p, _u32p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference harness not built: " + REF_SO)
        R = C.CDLL(REF_SO)
        R.ref_stitch.argtypes = [C.POINTER(C.c_void_p), _u32p, _u32p, _u32p, _u32p, C.c_uint32,
                                 C.c_void_p, C.c_uint32, C.c_uint64]
        R.ref_run_plan_sort.argtypes = [C.POINTER(C.c_void_p), _u32p, _u32p, C.c_uint32, _u32p,
                                        C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_double)]
        R.ref_sort_round.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_uint64]
        R.ref_run_plan_hash.argtypes = [C.POINTER(C.c_void_p), _u32p, _u32p, C.c_uint32, _u32p,
                                        C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_double)]
        _ref = R
    return _ref


def _u32arr(xs):
    a = (C.c_uint32 * len(xs))(*[int(x) for x in xs])
    return a


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


# ---------------------------------------------------------------------------
# C restatement
# ---------------------------------------------------------------------------
def plan_records(bw, split, col_order=None):
    """[(final_idx, start, end), ...] per bank (src/stitch_composer.cpp:568-612)."""
    ncols, nbanks = len(bw), len(split)
    col_order = list(range(ncols)) if col_order is None else list(col_order)
    rec = (_Record * (ncols + nbanks))()
    nrec = (C.c_uint32 * nbanks)()
    n = lib().orc_plan_records(_u32arr(bw), ncols, _u32arr(col_order), _u32arr(split), nbanks,
                               rec, nrec)
    if n < 0:
        raise ValueError(f"split {split} does not match widths {bw}")
    out, k = [], 0
    for b in range(nbanks):
        out.append([(rec[k + j].final_idx, rec[k + j].start, rec[k + j].end) for j in range(nrec[b])])
        k += nrec[b]
    return out


def bank_bytes(bits: int, hash_path: bool = False) -> int:
    return int(lib().orc_bank_bytes(bits, 1 if hash_path else 0))


def stitch(slices, bank_bytes_: int, n: int) -> np.ndarray:
    """slices: [(array, src_bits, start, end)]."""
    arr = (_Slice * len(slices))()
    keep = []
    for i, (a, bits, s, e) in enumerate(slices):
        a = np.ascontiguousarray(a)
        keep.append(a)
        arr[i] = _Slice(a.ctypes.data, a.dtype.itemsize, bits, s, e)
    out = np.zeros(n, dtype=np.dtype(f"u{bank_bytes_}"))
    _check(lib().orc_stitch(arr, len(slices), _ptr(out), bank_bytes_, n), "orc_stitch")
    return out


def sort_round(bank: np.ndarray, order=None, in_group=None, want_group=True):
    """Returns (order, group or None, sorted_keys, ngroups)."""
    n = bank.shape[0]
    order = np.zeros(n, np.uint32) if order is None else np.array(order, np.uint32, copy=True)
    out_group = np.zeros(n, np.uint32) if want_group else None
    keys = np.zeros_like(bank)
    ng = C.c_uint32(0)
    ig = None if in_group is None else np.ascontiguousarray(in_group, np.uint32)
    _check(lib().orc_sort_round(_ptr(np.ascontiguousarray(bank)), bank.dtype.itemsize, _ptr(order),
                                _ptr(ig), _ptr(out_group), _ptr(keys), n, C.byref(ng)),
           "orc_sort_round")
    return order, out_group, keys, ng.value


def hash_round(bank: np.ndarray, order=None, in_group=None, last_round=False):
    """Returns (order, out_group or None, group_idx, ngroups)."""
    n = bank.shape[0]
    order = np.zeros(n, np.uint32) if order is None else np.array(order, np.uint32, copy=True)
    out_group = None if last_round else np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    ng = C.c_uint32(0)
    ig = None if in_group is None else np.ascontiguousarray(in_group, np.uint32)
    _check(lib().orc_hash_round(_ptr(np.ascontiguousarray(bank)), bank.dtype.itemsize, _ptr(order),
                                _ptr(ig), _ptr(out_group), _ptr(idx), n, 1 if last_round else 0,
                                C.byref(ng)), "orc_hash_round")
    return order, out_group, idx, ng.value


def hash_unordered(bank: np.ndarray, in_group=None):
    """Returns (group ids in row order, ngroups)."""
    n = bank.shape[0]
    out = np.zeros(n, np.uint32)
    ng = C.c_uint32(0)
    ig = None if in_group is None else np.ascontiguousarray(in_group, np.uint32)
    _check(lib().orc_hash_unordered(_ptr(np.ascontiguousarray(bank)), bank.dtype.itemsize, _ptr(ig), _ptr(out), n,
                                    C.byref(ng)), "orc_hash_unordered")
    return out, ng.value


def _plan_args(cols, bw, split):
    cols = [np.ascontiguousarray(c) for c in cols]
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    cb = _u32arr([c.dtype.itemsize for c in cols])
    return cols, ptrs, cb, _u32arr(bw), _u32arr(split)


def run_plan_sort(cols, bw, split, col_order=None):
    """Whole sort plan; returns (order, group, ngroups).  col_order[k] is the
    column whose bits come k-th (None: 0..ncols-1)."""
    n = cols[0].shape[0]
    keep, ptrs, cb, bwa, spa = _plan_args(cols, bw, split)
    co = None if col_order is None else _u32arr(col_order)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = C.c_uint32(0)
    _check(lib().orc_run_plan_sort(ptrs, cb, bwa, len(cols), co, spa, len(split), n, _ptr(order),
                                   _ptr(group), C.byref(ng)), "orc_run_plan_sort")
    return order, group, ng.value


def run_plan_hash(cols, bw, split, col_order=None):
    """Whole hash plan; returns (order, group, ngroups); col_order as for
    run_plan_sort."""
    n = cols[0].shape[0]
    keep, ptrs, cb, bwa, spa = _plan_args(cols, bw, split)
    co = None if col_order is None else _u32arr(col_order)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = C.c_uint32(0)
    _check(lib().orc_run_plan_hash(ptrs, cb, bwa, len(cols), co, spa, len(split), n, _ptr(order),
                                   _ptr(group), C.byref(ng)), "orc_run_plan_hash")
    return order, group, ng.value


# ---------------------------------------------------------------------------
# reference harness (the reference's own code)
# ---------------------------------------------------------------------------
def ref_stitch(slices, bank_bytes_: int, n: int) -> np.ndarray:
    keep = [np.ascontiguousarray(a) for a, *_ in slices]
    ptrs = (C.c_void_p * len(slices))(*[a.ctypes.data for a in keep])
    out = np.zeros(n, dtype=np.dtype(f"u{bank_bytes_}"))
    _check(ref().ref_stitch(ptrs, _u32arr([a.dtype.itemsize for a in keep]),
                            _u32arr([s[1] for s in slices]), _u32arr([s[2] for s in slices]),
                            _u32arr([s[3] for s in slices]), len(slices), _ptr(out), bank_bytes_, n),
           "ref_stitch")
    return out


def ref_run_plan_sort(cols, bw, split, final_groups=True):
    """Returns (order, group or None, seconds).  order is the reference's raw
    (unstable) order; canonicalise ties before comparing."""
    n = cols[0].shape[0]
    keep, ptrs, cb, bwa, spa = _plan_args(cols, bw, split)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32) if final_groups else None
    secs = C.c_double(0)
    _check(ref().ref_run_plan_sort(ptrs, cb, bwa, len(cols), spa, len(split), n, _ptr(order),
                                   _ptr(group), 1 if final_groups else 0, C.byref(secs)),
           "ref_run_plan_sort")
    return order, group, secs.value


def ref_sort_round(bank: np.ndarray, bits: int, order=None, in_group=None):
    n = bank.shape[0]
    order = np.zeros(n, np.uint32) if order is None else np.array(order, np.uint32, copy=True)
    group = np.zeros(n, np.uint32)
    ig = None if in_group is None else np.ascontiguousarray(in_group, np.uint32)
    _check(ref().ref_sort_round(_ptr(np.ascontiguousarray(bank)), bank.dtype.itemsize, bits,
                                _ptr(order), _ptr(ig), _ptr(group), n), "ref_sort_round")
    return order, group


def ref_run_plan_hash(cols, bw, split):
    n = cols[0].shape[0]
    keep, ptrs, cb, bwa, spa = _plan_args(cols, bw, split)
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    secs = C.c_double(0)
    _check(ref().ref_run_plan_hash(ptrs, cb, bwa, len(cols), spa, len(split), n, _ptr(order),
                                   _ptr(group), C.byref(secs)), "ref_run_plan_hash")
    return order, group, secs.value


def canonicalize(order: np.ndarray, group: np.ndarray) -> np.ndarray:
    """Sort oids ascending inside each group (groups are contiguous runs)."""
    g = np.asarray(group, np.uint64)
    if g.size and np.all(g[1:] >= g[:-1]):
        # ids ascend with the position: one sort of (group << 32 | oid)
        key = (g << np.uint64(32)) | np.asarray(order, np.uint64)
        key.sort()
        return (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    idx = np.lexsort((order, group))
    return order[idx]
