"""ctypes binding of ``libfmcs.so`` (include/fmcs_capi.h).

This is the Python face of the drop-in boundary: every method is one C-ABI
call.  Arrays may be numpy arrays (host memory; the library stages them) or
CUDA tensors / objects exposing ``data_ptr()`` (device memory, used in place).

There is no CPU fallback: if the shared library is missing or no GPU is
visible, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmcs.so")

FMCS_OK = 0
FMCS_E_INVAL = -1
FMCS_E_OOM = -2
FMCS_E_TIMEOUT = -3
FMCS_E_CUDA = -4

# Every symbol include/fmcs_capi.h declares.
EXPORTS = (
    "fmcs_create", "fmcs_destroy", "fmcs_last_error", "fmcs_synchronize", "fmcs_stream",
    "fmcs_workspace_bytes", "fmcs_stitch", "fmcs_gather", "fmcs_sort_round", "fmcs_hash_round",
    "fmcs_run_plan", "fmcs_run_plan_desc", "fmcs_profile", "fmcs_profile_report", "fmcs_launch_count",
    "fmcs_group_ids_noalloc", "fmcs_shift_left", "fmcs_assemble", "fmcs_hash_round_unordered",
    "fmcs_sort_round_plain", "fmcs_optimize_plan", "fmcs_estimate_plan", "fmcs_set_tuning", "fmcs_get_tuning", "fmcs_run_batch",
    "fmcs_server_create", "fmcs_server_submit", "fmcs_server_wait", "fmcs_server_load", "fmcs_server_destroy",
    "fmcs_graph_create", "fmcs_graph_launch", "fmcs_graph_stream", "fmcs_graph_destroy", "fmcs_graph_kernels",
    "fmcs_storage_bytes", "fmcs_text_header", "fmcs_read_columns_text", "fmcs_write_columns_text",
    "fmcs_group_aggregate", "fmcs_selftest_wait", "fmcs_graph_create_hash",
)


class FmcsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fmcs error {code}: {msg}")
        self.code = code


class Instance(C.Structure):
    _fields_ = [("row_off", C.c_uint64), ("n", C.c_uint64)]


class Request(C.Structure):
    _fields_ = [("cols", C.POINTER(C.c_void_p)), ("col_bytes", C.POINTER(C.c_uint32)),
                ("bw", C.POINTER(C.c_uint32)), ("ncols", C.c_uint32), ("split", C.POINTER(C.c_uint32)),
                ("nbanks", C.c_uint32), ("cardinality", C.POINTER(C.c_uint64)), ("n", C.c_uint64),
                ("hash", C.c_int), ("order_out", C.c_void_p), ("group_out", C.c_void_p)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("ngroups", C.c_uint32), ("batched_with", C.c_uint32),
                ("queue_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double)]


class Slice(C.Structure):
    _fields_ = [("src", C.c_void_p), ("src_bytes", C.c_uint32), ("src_bits", C.c_uint32),
                ("start", C.c_uint32), ("end", C.c_uint32)]


_lib = None


def load(path: str = LIB_PATH):
    """Load libfmcs.so and declare its signatures (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run __graft_entry__.build() (nvcc, sm_100a)")
    L = C.CDLL(path)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    u32p = C.POINTER(C.c_uint32)
    L.fmcs_create.argtypes = [C.POINTER(vp), i32, C.c_size_t]
    L.fmcs_destroy.argtypes = [vp]
    L.fmcs_destroy.restype = None
    L.fmcs_last_error.argtypes = [vp]
    L.fmcs_last_error.restype = C.c_char_p
    L.fmcs_synchronize.argtypes = [vp]
    L.fmcs_stream.argtypes = [vp]
    L.fmcs_stream.restype = vp
    L.fmcs_workspace_bytes.argtypes = [vp]
    L.fmcs_workspace_bytes.restype = C.c_size_t
    L.fmcs_stitch.argtypes = [vp, C.POINTER(Slice), u32, vp, u32, u64]
    L.fmcs_gather.argtypes = [vp, vp, u32, vp, vp, u64]
    L.fmcs_sort_round.argtypes = [vp, vp, u32, u32, vp, vp, vp, vp, u64, u32p]
    L.fmcs_hash_round.argtypes = [vp, vp, u32, vp, vp, vp, u64, i32, u32p]
    L.fmcs_run_plan.argtypes = [vp, C.POINTER(vp), u32p, u32p, u32, u32p, u32p, u32, u64, i32,
                                vp, vp, u32p]
    L.fmcs_group_aggregate.argtypes = [vp, vp, u32, i32, vp, vp, u64, u32, vp, vp, vp, vp]
    L.fmcs_storage_bytes.argtypes = [u32]
    L.fmcs_storage_bytes.restype = u32
    L.fmcs_text_header.argtypes = [C.c_char_p, C.POINTER(u64), C.POINTER(u32)]
    L.fmcs_read_columns_text.argtypes = [C.c_char_p, i32, u32, u32p, u64, C.POINTER(vp), C.POINTER(u64)]
    L.fmcs_write_columns_text.argtypes = [C.c_char_p, i32, u32, u64, C.POINTER(vp), u32p]
    L.fmcs_run_plan_desc.argtypes = [vp, C.POINTER(vp), u32p, u32p, u32, u32p, C.POINTER(C.c_uint8), u32p, u32,
                                     u64, i32, vp, vp, u32p]
    L.fmcs_profile.argtypes = [vp, i32]
    L.fmcs_profile_report.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.fmcs_selftest_wait.argtypes = [vp, u32]
    L.fmcs_launch_count.argtypes = [vp]
    L.fmcs_launch_count.restype = C.c_ulonglong
    L.fmcs_group_ids_noalloc.argtypes = [vp, vp, u32, vp, vp, u64, u32p]
    L.fmcs_shift_left.argtypes = [vp, vp, u32, u64, u32]
    L.fmcs_assemble.argtypes = [vp, vp, u32, u64, C.POINTER(Slice)]
    L.fmcs_hash_round_unordered.argtypes = [vp, vp, u32, vp, vp, u64, u32p]
    L.fmcs_sort_round_plain.argtypes = [vp, vp, u32, u32, vp, vp, vp, vp, u64, u32p]
    L.fmcs_run_batch.argtypes = [vp, C.POINTER(vp), u32p, u32p, u32, u32p, u32, C.POINTER(Instance), u32, u64,
                                 vp, vp, u32p]
    L.fmcs_graph_create.argtypes = [vp, C.POINTER(vp), u32p, u32p, u32, u32p, u32p, u32, u64, vp, vp, C.POINTER(vp)]
    L.fmcs_graph_create_hash.argtypes = [vp, C.POINTER(vp), u32p, u32p, u32, u32p, u32p, u32, u64, vp, vp,
                                         C.POINTER(vp)]
    L.fmcs_graph_launch.argtypes = [vp, u32p]
    L.fmcs_graph_stream.argtypes = [vp]
    L.fmcs_graph_stream.restype = vp
    L.fmcs_graph_kernels.argtypes = [vp]
    L.fmcs_graph_destroy.argtypes = [vp]
    L.fmcs_graph_destroy.restype = None
    L.fmcs_server_create.argtypes = [C.POINTER(vp), i32, C.c_size_t, u32, u64]
    L.fmcs_server_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(C.c_uint64)]
    L.fmcs_server_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(Result)]
    L.fmcs_server_load.argtypes = [vp, C.POINTER(C.c_size_t), u32p, u32p]
    L.fmcs_server_destroy.argtypes = [vp]
    L.fmcs_server_destroy.restype = None
    L.fmcs_set_tuning.argtypes = [vp, C.c_char_p, C.c_longlong]
    L.fmcs_get_tuning.argtypes = [vp, C.c_char_p]
    L.fmcs_get_tuning.restype = C.c_longlong
    L.fmcs_optimize_plan.argtypes = [u32p, C.POINTER(C.c_uint64), u32p, u32, u64, i32, u32p, u32, u32p, u32p,
                                     C.POINTER(C.c_double)]
    L.fmcs_estimate_plan.argtypes = [u32p, C.POINTER(C.c_uint64), u32p, u32, u64, u32p, u32p, u32,
                                     C.POINTER(C.c_double)]
    _lib = L
    return L


def _addr(a) -> Optional[int]:
    """Address of a numpy array (host) or a device tensor (data_ptr)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return int(a.ctypes.data)
    raise TypeError(f"unsupported array type {type(a)}")


def _itemsize(a) -> int:
    if hasattr(a, "element_size"):
        return int(a.element_size())
    return int(a.dtype.itemsize)


def _len(a) -> int:
    return int(a.shape[0])


def _u32arr(xs: Sequence[int]):
    return (C.c_uint32 * len(xs))(*[int(x) for x in xs])


def group_ids_noalloc(keys, out_group, in_group=None, stream: int = 0) -> int:
    """fmcs_group_ids_noalloc: dense group ids of sorted device keys with no
    device allocation (scratch in the library's static device array, at most
    67,108,864 rows).  keys / in_group / out_group must be device tensors;
    returns the group count."""
    L = load()
    ng = C.c_uint32(0)
    rc = L.fmcs_group_ids_noalloc(C.c_void_p(stream or None), _addr(keys), _itemsize(keys),
                                  _addr(in_group), _addr(out_group), _len(keys), C.byref(ng))
    if rc != FMCS_OK:
        raise FmcsError(rc, "fmcs_group_ids_noalloc failed")
    return ng.value


def storage_bytes(bw: int) -> int:
    """Bytes per value of a column of declared width bw (the reference's
    width -> type mapping: <= 16 bits u16, <= 32 u32, else u64)."""
    return int(load().fmcs_storage_bytes(int(bw)))


def text_header(path: str):
    """(row count, column count) of a dataset file with the TPC-H header."""
    n, c = C.c_uint64(0), C.c_uint32(0)
    rc = load().fmcs_text_header(str(path).encode(), C.byref(n), C.byref(c))
    if rc != FMCS_OK:
        raise FmcsError(rc, f"fmcs_text_header failed on {path}")
    return n.value, c.value


def read_columns_text(path: str, bw, nrows: int = None, header: bool = False, cardinality: bool = True):
    """The reference's text dataset (column after column; header = the TPC-H
    variant, whose row count is used when nrows is None).  Returns the columns
    as numpy arrays in their storage widths and, with cardinality, each
    column's number of distinct values."""
    if nrows is None:
        if not header:
            raise ValueError("nrows is required for a file without a header")
        nrows, _ = text_header(path)
    dts = {2: np.uint16, 4: np.uint32, 8: np.uint64}
    cols = [np.empty(nrows, dts[storage_bytes(w)]) for w in bw]
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    card = (C.c_uint64 * len(cols))()
    rc = load().fmcs_read_columns_text(str(path).encode(), 1 if header else 0, len(cols), _u32arr(bw), nrows, ptrs,
                                       card if cardinality else None)
    if rc != FMCS_OK:
        raise FmcsError(rc, f"fmcs_read_columns_text failed on {path}")
    return cols, ([int(x) for x in card] if cardinality else None)


def write_columns_text(path: str, cols, header: bool = False):
    """Writes numpy columns (2, 4 or 8 bytes per value) in the same format."""
    cols = [np.ascontiguousarray(c) for c in cols]
    nrows = cols[0].shape[0]
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    rc = load().fmcs_write_columns_text(str(path).encode(), 1 if header else 0, len(cols), nrows, ptrs,
                                        _u32arr([c.dtype.itemsize for c in cols]))
    if rc != FMCS_OK:
        raise FmcsError(rc, f"fmcs_write_columns_text failed on {path}")


def effective_cardinality(counts) -> int:
    """The cardinality to give the cost model for a skewed column: n^2 / sum of
    count^2 over its values' row counts, the number of EQUAL groups with the
    same row-weighted mean group size (the size of the group the average row
    sits in).  The model assumes equal groups; for uniform columns this is the
    distinct count, for a Zipf(1.0) column over 2^20 codes in 67M rows it is
    about 127 against 1,046,545 distinct values."""
    c = np.asarray(counts, dtype=np.float64)
    n = c.sum()
    sq = float(np.dot(c, c))
    return max(1, int(round(n * n / sq))) if sq > 0 else 1


def estimate_plan(bw, cardinality, col_bytes, n: int, split, col_order=None) -> float:
    """The cost model's estimated ms for one given plan (fmcs_estimate_plan)."""
    L = load()
    k = len(bw)
    est = C.c_double(0)
    rc = L.fmcs_estimate_plan(_u32arr(bw), (C.c_uint64 * k)(*[int(c) for c in cardinality]), _u32arr(col_bytes),
                              k, n, _u32arr(col_order) if col_order is not None else None, _u32arr(split),
                              len(split), C.byref(est))
    if rc != FMCS_OK:
        raise FmcsError(rc, "fmcs_estimate_plan failed")
    return est.value


def optimize_plan(bw, cardinality, col_bytes, n: int, ordered: bool = True):
    """Cost-model plan search; returns (split, column order, estimated ms)."""
    L = load()
    k = len(bw)
    split = (C.c_uint32 * 64)()
    nb = C.c_uint32(0)
    order = (C.c_uint32 * k)()
    est = C.c_double(0)
    rc = L.fmcs_optimize_plan(_u32arr(bw), (C.c_uint64 * k)(*[int(c) for c in cardinality]), _u32arr(col_bytes),
                              k, n, 1 if ordered else 0, split, 64, C.byref(nb), order, C.byref(est))
    if rc != FMCS_OK:
        raise FmcsError(rc, "fmcs_optimize_plan failed")
    return [split[i] for i in range(nb.value)], [order[i] for i in range(k)], est.value


class Context:
    """An fmcs_ctx: one CUDA stream and a reusable device workspace."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._L = load()
        h = C.c_void_p()
        rc = self._L.fmcs_create(C.byref(h), device, hbm_budget_bytes)
        if rc != FMCS_OK:
            raise FmcsError(rc, f"fmcs_create failed on device {device}")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.fmcs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc: int):
        if rc != FMCS_OK:
            msg = self._L.fmcs_last_error(self._h)
            raise FmcsError(rc, msg.decode() if msg else "")

    def synchronize(self):
        self._check(self._L.fmcs_synchronize(self._h))

    @property
    def stream(self) -> int:
        return int(self._L.fmcs_stream(self._h) or 0)

    def profile(self, enable: bool = True):
        self._check(self._L.fmcs_profile(self._h, 1 if enable else 0))

    def profile_report(self) -> dict:
        """Per-kernel {launches, ms} since the last report (synchronizes)."""
        import json
        buf = C.create_string_buffer(1 << 16)
        self._check(self._L.fmcs_profile_report(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def selftest_wait(self, polls: int) -> int:
        """fmcs_selftest_wait: a bounded device wait on a word nothing writes;
        returns the status code (FMCS_E_TIMEOUT when the wait gave up)."""
        return int(self._L.fmcs_selftest_wait(self._h, int(polls)))

    def launch_count(self) -> int:
        return int(self._L.fmcs_launch_count(self._h))

    def set_tuning(self, key: str, value: int):
        self._check(self._L.fmcs_set_tuning(self._h, key.encode(), int(value)))

    def get_tuning(self, key: str) -> int:
        return int(self._L.fmcs_get_tuning(self._h, key.encode()))

    def workspace_bytes(self) -> int:
        return int(self._L.fmcs_workspace_bytes(self._h))

    # -- (a) --------------------------------------------------------------
    def stitch(self, slices, bank, n: Optional[int] = None):
        """slices: [(array, src_bits, start, end)]; bank: output array."""
        n = _len(bank) if n is None else n
        arr = (Slice * len(slices))()
        for i, (a, bits, s, e) in enumerate(slices):
            arr[i] = Slice(_addr(a), _itemsize(a), bits, s, e)
        self._check(self._L.fmcs_stitch(self._h, arr, len(slices), _addr(bank), _itemsize(bank), n))
        return bank

    def shift_left(self, bank, nbits: int):
        """bank <<= nbits in place (ShiftLeftBatch)."""
        self._check(self._L.fmcs_shift_left(self._h, _addr(bank), _itemsize(bank), _len(bank), nbits))
        return bank

    def assemble(self, bank, src, src_bits: int, start: int, end: int):
        """bank |= slice of src (AssembleFromColumn)."""
        sl = Slice(_addr(src), _itemsize(src), src_bits, start, end)
        self._check(self._L.fmcs_assemble(self._h, _addr(bank), _itemsize(bank), _len(bank), C.byref(sl)))
        return bank

    # -- (c) --------------------------------------------------------------
    def gather(self, bank, order, out):
        self._check(self._L.fmcs_gather(self._h, _addr(bank), _itemsize(bank), _addr(order),
                                        _addr(out), _len(order)))
        return out

    # -- (b)+(d) ----------------------------------------------------------
    def sort_round(self, bank, key_bits: int, order, in_group=None, out_group=None,
                   sorted_bank=None) -> int:
        ng = C.c_uint32(0)
        self._check(self._L.fmcs_sort_round(self._h, _addr(bank), _itemsize(bank), key_bits,
                                            _addr(order), _addr(in_group), _addr(out_group),
                                            _addr(sorted_bank), _len(bank), C.byref(ng)))
        return ng.value

    def sort_round_plain(self, bank, key_bits: int, order, in_group=None, out_group=None,
                         sorted_bank=None) -> int:
        """The unsegmented comparator round (full-array LSD passes)."""
        ng = C.c_uint32(0)
        self._check(self._L.fmcs_sort_round_plain(self._h, _addr(bank), _itemsize(bank), key_bits,
                                                  _addr(order), _addr(in_group), _addr(out_group),
                                                  _addr(sorted_bank), _len(bank), C.byref(ng)))
        return ng.value

    def hash_round_unordered(self, bank, out_group, in_group=None) -> int:
        ng = C.c_uint32(0)
        self._check(self._L.fmcs_hash_round_unordered(self._h, _addr(bank), _itemsize(bank), _addr(in_group),
                                                      _addr(out_group), _len(bank), C.byref(ng)))
        return ng.value

    # -- (e) --------------------------------------------------------------
    def hash_round(self, bank, order, in_group=None, out_group=None, last_round=False) -> int:
        ng = C.c_uint32(0)
        self._check(self._L.fmcs_hash_round(self._h, _addr(bank), _itemsize(bank), _addr(order),
                                            _addr(in_group), _addr(out_group), _len(bank),
                                            1 if last_round else 0, C.byref(ng)))
        return ng.value

    # -- CUDA graph of a whole plan -----------------------------------------
    def plan_graph(self, cols, bw, split, order_out, group_out=None, col_order=None,
                   hash: bool = False) -> "PlanGraph":
        """A CUDA graph of the plan (fmcs_graph_create, or with hash the
        hash-grouping plan: fmcs_graph_create_hash)."""
        return PlanGraph(self, cols, bw, split, order_out, group_out, col_order, hash)

    # -- many instances ----------------------------------------------------
    def run_batch(self, cols, bw, split, sizes, order_out, group_out=None):
        """sizes[k] rows per instance, concatenated in the column arrays; returns
        the per-instance group counts."""
        k = len(sizes)
        inst = (Instance * k)()
        off = 0
        for i, s in enumerate(sizes):
            inst[i] = Instance(off, int(s))
            off += int(s)
        ptrs = (C.c_void_p * len(cols))(*[_addr(c) for c in cols])
        counts = np.zeros(k, np.uint32)
        self._check(self._L.fmcs_run_batch(self._h, ptrs, _u32arr([_itemsize(c) for c in cols]), _u32arr(bw),
                                           len(cols), _u32arr(split), len(split), inst, k, off, _addr(order_out),
                                           _addr(group_out), counts.ctypes.data_as(C.POINTER(C.c_uint32))))
        return counts

    def group_aggregate(self, payload, order, group, ngroups: int, count=None, sum=None, min=None, max=None,
                        signed: bool = False):
        """fmcs_group_aggregate: per-group count / sum / min / max (int64 device
        tensors of ngroups entries, any may be None) of payload[order[i]] over
        the sorted positions i of each group."""
        self._check(self._L.fmcs_group_aggregate(self._h, _addr(payload), _itemsize(payload), 1 if signed else 0,
                                                 _addr(order), _addr(group), _len(order), int(ngroups), _addr(count),
                                                 _addr(sum), _addr(min), _addr(max)))

    # -- whole plan ---------------------------------------------------------
    def run_plan(self, cols, bw, split, order_out, group_out=None, col_order=None,
                 hash: bool = False, descending=None) -> int:
        """descending[c] true sorts column c in descending order (fmcs_run_plan_desc)."""
        n = _len(cols[0])
        ptrs = (C.c_void_p * len(cols))(*[_addr(c) for c in cols])
        ng = C.c_uint32(0)
        co = None if col_order is None else _u32arr(col_order)
        if descending is None:
            self._check(self._L.fmcs_run_plan(self._h, ptrs, _u32arr([_itemsize(c) for c in cols]),
                                              _u32arr(bw), len(cols), co, _u32arr(split), len(split), n,
                                              1 if hash else 0, _addr(order_out), _addr(group_out),
                                              C.byref(ng)))
        else:
            desc = (C.c_uint8 * len(cols))(*[1 if d else 0 for d in descending])
            self._check(self._L.fmcs_run_plan_desc(self._h, ptrs, _u32arr([_itemsize(c) for c in cols]),
                                                   _u32arr(bw), len(cols), co, desc, _u32arr(split), len(split),
                                                   n, 1 if hash else 0, _addr(order_out), _addr(group_out),
                                                   C.byref(ng)))
        return ng.value


class PlanGraph:
    """fmcs_graph: a sort plan captured once, replayed with launch()."""

    def __init__(self, ctx: "Context", cols, bw, split, order_out, group_out=None, col_order=None,
                 hash: bool = False):
        self._L = load()
        self._ctx = ctx
        n = _len(cols[0])
        self._keep = (cols, order_out, group_out)
        ptrs = (C.c_void_p * len(cols))(*[_addr(c) for c in cols])
        co = None if col_order is None else _u32arr(col_order)
        h = C.c_void_p()
        create = self._L.fmcs_graph_create_hash if hash else self._L.fmcs_graph_create
        rc = create(ctx.handle, ptrs, _u32arr([_itemsize(c) for c in cols]), _u32arr(bw),
                    len(cols), co, _u32arr(split), len(split), n, _addr(order_out),
                    _addr(group_out), C.byref(h))
        ctx._check(rc)
        self._h = h

    def launch(self) -> int:
        ng = C.c_uint32(0)
        rc = self._L.fmcs_graph_launch(self._h, C.byref(ng))
        if rc != FMCS_OK:
            raise FmcsError(rc, "fmcs_graph_launch failed")
        return ng.value

    @property
    def stream(self) -> int:
        return int(self._L.fmcs_graph_stream(self._h) or 0)

    def kernels(self) -> int:
        """Kernel nodes of the graph (each loop body counted once)."""
        return int(self._L.fmcs_graph_kernels(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.fmcs_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """fmcs_server (include/fmcs_server.h): execution slots with their own
    streams, admission against an HBM budget, continuous batching of small
    compatible requests."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 << 30, slots: int = 4,
                 batch_rows_max: int = 1 << 20):
        self._L = load()
        h = C.c_void_p()
        rc = self._L.fmcs_server_create(C.byref(h), device, hbm_budget_bytes, slots, batch_rows_max)
        if rc != FMCS_OK:
            raise FmcsError(rc, "fmcs_server_create failed")
        self._h = h
        self._keep = {}

    def submit(self, cols, bw, order_out, group_out=None, split=None, cardinality=None, hash=False) -> int:
        n = _len(cols[0])
        ptrs = (C.c_void_p * len(cols))(*[_addr(c) for c in cols])
        cb = _u32arr([_itemsize(c) for c in cols])
        bwa = _u32arr(bw)
        spl = _u32arr(split) if split else None
        card = (C.c_uint64 * len(cols))(*[int(x) for x in cardinality]) if cardinality else None
        req = Request(ptrs, cb, bwa, len(cols), spl, len(split) if split else 0, card, n, 1 if hash else 0,
                      _addr(order_out), _addr(group_out))
        t = C.c_uint64(0)
        rc = self._L.fmcs_server_submit(self._h, C.byref(req), C.byref(t))
        if rc != FMCS_OK:
            raise FmcsError(rc, "fmcs_server_submit failed")
        self._keep[t.value] = (ptrs, cb, bwa, spl, card, cols, order_out, group_out)
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0) -> dict:
        r = Result()
        rc = self._L.fmcs_server_wait(self._h, ticket, timeout_s, C.byref(r))
        if rc != FMCS_OK:
            raise FmcsError(rc, "fmcs_server_wait failed")
        self._keep.pop(ticket, None)
        return {"status": r.status, "ngroups": r.ngroups, "batched_with": r.batched_with,
                "queue_ms": r.queue_ms, "run_ms": r.run_ms, "total_ms": r.total_ms}

    def load(self):
        a, q, r = C.c_size_t(0), C.c_uint32(0), C.c_uint32(0)
        self._L.fmcs_server_load(self._h, C.byref(a), C.byref(q), C.byref(r))
        return a.value, q.value, r.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.fmcs_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
