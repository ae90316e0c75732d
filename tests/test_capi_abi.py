"""The C-ABI library exists, loads, and exports every symbol that
include/*.h declares; the Python binding declares the same set.  No compute
calls: this runs without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

from fastmulticolsort_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        syms |= set(re.findall(r"FMCS_API[^;(]*?\b(fmcs_\w+)\s*\(", txt))
    return syms


def test_library_built():
    assert os.path.exists(capi.LIB_PATH), "run __graft_entry__.build()"


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 11
    lib = ctypes.CDLL(capi.LIB_PATH)
    for s in sorted(syms):
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\b(fmcs_\w+)$", out, re.M))
    assert syms <= exported
    assert set(capi.EXPORTS) == syms


def test_binding_loads():
    L = capi.load()
    assert L.fmcs_create is not None


def test_no_silent_fallback_without_gpu():
    # On a machine without a visible GPU the context must fail loudly.
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    with pytest.raises(capi.FmcsError):
        capi.Context(0)
