"""B200-native multi-column sort path of FastMultiColSort.

The product is ``libfmcs.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/fmcs_capi.h``) and the C++ host classes in ``include/fmcs/``; this
package holds their sources (``csrc/``), the build recipe, the ctypes binding
(``capi``) and the seeded workload generators (``workloads``).
"""
from .build import build_native, LIB_PATH  # noqa: F401

__all__ = ["build_native", "LIB_PATH"]
