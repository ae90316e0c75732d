"""Build recipe of the native library: ``make`` over ``csrc/Makefile`` (nvcc
``-gencode arch=compute_100a,code=sm_100a -lineinfo``).  The library is built
in-tree (``fastmulticolsort_b200/libfmcs.so``) so that it travels with the
repository snapshot."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmcs.so")


def build_native(jobs: int = 8, verbose: bool = False) -> str:
    cmd = ["make", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return LIB_PATH
