"""magma_b200 -- B200-native batched small-matrix dense solvers behind MAGMA's C API.

The product is the shared library ``libmagma_b200.so`` (C ABI in
``include/magma_b200.h``). This package holds its CUDA/C++ sources
(``csrc/``), the in-tree build (``build.py``), a ctypes binding (``_lib.py``)
and thin torch-facing helpers used by the tests, the benchmark and the
request loop. The helpers only marshal device pointers; every computation
runs in the library's kernels.
"""
from __future__ import annotations

import os

# The library's queues use more streams than the driver's default 8 hardware work
# queues; ask for 32 before any CUDA context exists (a value already set is kept).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _lib  # noqa: E402
from .api import (HostDgesv, HostDsgesv, Queue, VarBatch, dgeqrf_batched, dgerbt_batched, dgesv_batched, dgesv_nopiv_batched,  # noqa: E402
                  dgesv_rbt_batched, dgesv_vbatched, dgetrf_batched, dgetrf_nopiv_batched, dgetri_outofplace_batched,
                  dgetrs_batched, dgetrs_nopiv_batched, dposv_batched, dposv_vbatched, dpotrf_batched,
                  dpotrs_batched, dsgesv_batched, dsposv_vbatched, gemm_batched, gemm_vbatched, ptr_array,
                  syrk_vbatched, tri_vbatched)

__all__ = ["HostDgesv", "HostDsgesv", "Queue", "VarBatch", "ptr_array", "dgetrf_batched", "dgetrs_batched", "dgesv_batched", "dpotrf_batched",
           "dpotrs_batched", "dposv_batched", "dposv_vbatched", "dsgesv_batched", "dgesv_vbatched", "dsposv_vbatched",
           "dgetri_outofplace_batched", "dgetrf_nopiv_batched", "dgetrs_nopiv_batched", "dgesv_nopiv_batched",
           "dgerbt_batched", "dgesv_rbt_batched", "dgeqrf_batched", "gemm_batched", "gemm_vbatched", "syrk_vbatched",
           "tri_vbatched", "load"]


def load():
    """Load libmagma_b200.so (raises if it has not been built)."""
    return _lib.load()
