"""ctypes binding of libmagma_b200.so (the C ABI declared in include/magma_b200.h).

The shared library is built in-tree by ``python -m magma_b200.build``. There is
no fallback: if the library is missing or fails to load, importing the
bindings raises, so nothing can silently run on another implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmagma_b200.so"

magma_int_t = C.c_int
_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_f = C.c_float
_s = C.c_char_p
_sz = C.c_size_t

MagmaNoTrans, MagmaTrans, MagmaConjTrans = 111, 112, 113
MagmaUpper, MagmaLower, MagmaFull = 121, 122, 123
MagmaNonUnit, MagmaUnit = 131, 132
MagmaLeft, MagmaRight = 141, 142
MagmaFalse, MagmaTrue = 0, 1

MAGMA_SUCCESS = 0
MAGMA_ERR_NOT_SUPPORTED = -103
MAGMA_ERR_ILLEGAL_VALUE = -104
MAGMA_ERR_DEVICE_ALLOC = -113

# name -> (restype, argtypes). Every symbol declared in include/magma_b200.h
# appears here; tests check the two lists agree.
SIGNATURES: dict[str, tuple] = {
    # runtime
    "magma_init": (_i, []),
    "magma_finalize": (_i, []),
    "magma_strerror": (_s, [_i]),
    "magma_xerbla": (None, [_s, _i]),
    "magma_getdevice": (None, [C.POINTER(_i)]),
    "magma_setdevice": (None, [_i]),
    "magma_malloc": (_i, [C.POINTER(_p), _sz]),
    "magma_free_internal": (_i, [_p, _s, _s, _i]),
    "magma_malloc_pinned": (_i, [C.POINTER(_p), _sz]),
    "magma_free_pinned_internal": (_i, [_p, _s, _s, _i]),
    "magma_queue_create_internal": (None, [_i, C.POINTER(_p), _s, _s, _i]),
    "magma_queue_create_from_cuda_internal": (None, [_i, _p, _p, _p, C.POINTER(_p), _s, _s, _i]),
    "magma_queue_destroy_internal": (None, [_p, _s, _s, _i]),
    "magma_queue_sync_internal": (None, [_p, _s, _s, _i]),
    "magma_queue_get_device": (_i, [_p]),
    "magma_queue_get_cuda_stream": (_p, [_p]),
    "magma_queue_reserve_workspace": (_i, [_p, _sz]),
    "magma_b200_queue_set_workspace_limit": (_i, [_p, _sz]),
    "magma_b200_stage_timing": (_i, [_p, _i]),
    "magma_b200_stage_times": (_i, [_p, _p, _i]),
    "magma_b200_debug_tc_wait_limit": (None, [C.c_longlong]),
    "magma_setvector_internal": (None, [_i, _i, _p, _i, _p, _i, _p, _s, _s, _i]),
    "magma_getvector_internal": (None, [_i, _i, _p, _i, _p, _i, _p, _s, _s, _i]),
    "magma_setvector_async_internal": (None, [_i, _i, _p, _i, _p, _i, _p, _s, _s, _i]),
    "magma_getvector_async_internal": (None, [_i, _i, _p, _i, _p, _i, _p, _s, _s, _i]),
    "magma_dset_pointer": (None, [_p, _p, _i, _i, _i, _i, _i, _p]),
    "magma_sset_pointer": (None, [_p, _p, _i, _i, _i, _i, _i, _p]),
    "magma_iset_pointer": (None, [_p, _p, _i, _i, _i, _i, _i, _p]),
    # batched LU
    "magma_dgetrf_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p]),
    "magma_dgetrs_batched": (_i, [_i, _i, _i, _p, _i, _p, _p, _i, _i, _p]),
    "magma_dgesv_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p, _i, _p]),
    "magma_dgetrf_vbatched": (_i, [_p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dgetrf_vbatched_max_nocheck": (_i, [_p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magma_dgetrs_vbatched": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dgetrs_vbatched_max_nocheck": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magma_dgesv_vbatched": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dgesv_vbatched_max_nocheck": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magma_dgetri_outofplace_batched": (_i, [_i, _p, _i, _p, _p, _i, _p, _i, _p]),
    "magma_dgetrf_nopiv_batched": (_i, [_i, _i, _p, _i, _p, _i, _p]),
    "magma_dgetrs_nopiv_batched": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _i, _p]),
    "magma_dgesv_nopiv_batched": (_i, [_i, _i, _p, _i, _p, _i, _p, _i, _p]),
    "magma_dgerbt_batched": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _p, _p, _i, _p]),
    "magma_dgeqrf_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p]),
    "magma_dgesv_rbt_batched": (_i, [_i, _i, _p, _i, _p, _i, _p, _i, _p]),
    "magma_sgetrf_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p]),
    "magma_sgetrs_batched": (_i, [_i, _i, _i, _p, _i, _p, _p, _i, _i, _p]),
    "magma_sgesv_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p, _i, _p]),
    "magma_dsgesv_batched": (_i, [_i, _i, _p, _i, _p, _p, _i, _p, _i, _p, _p, _i, _p]),
    # batched Cholesky
    "magma_dpotrf_batched": (_i, [_i, _i, _p, _i, _p, _i, _p]),
    "magma_dpotrs_batched": (_i, [_i, _i, _i, _p, _i, _p, _i, _i, _p]),
    "magma_dposv_batched": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _i, _p]),
    "magma_dpotrf_vbatched": (_i, [_i, _p, _p, _p, _p, _i, _p]),
    "magma_dpotrf_vbatched_max_nocheck": (_i, [_i, _p, _p, _p, _p, _i, _i, _p]),
    "magma_dpotrf_vbatched_max_nocheck_noalloc": (_i, [_i, _p, _p, _p, _p, _i, _i, _p]),
    "magma_dpotrs_vbatched": (_i, [_i, _p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dpotrs_vbatched_max_nocheck": (_i, [_i, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magma_dposv_vbatched": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dposv_vbatched_max_nocheck": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    # batched gemm
    "magmablas_dgemm_batched": (None, [_i, _i, _i, _i, _i, _d, _p, _i, _p, _i, _d, _p, _i, _i, _p]),
    "magma_dgemm_batched": (None, [_i, _i, _i, _i, _i, _d, _p, _i, _p, _i, _d, _p, _i, _i, _p]),
    "magmablas_sgemm_batched": (None, [_i, _i, _i, _i, _i, _f, _p, _i, _p, _i, _f, _p, _i, _i, _p]),
    "magma_sgemm_batched": (None, [_i, _i, _i, _i, _i, _f, _p, _i, _p, _i, _f, _p, _i, _i, _p]),
    "magmablas_dgemm_vbatched": (None, [_i, _i, _p, _p, _p, _d, _p, _p, _p, _p, _d, _p, _p, _i, _p]),
    "magmablas_dgemm_vbatched_max_nocheck": (None, [_i, _i, _p, _p, _p, _d, _p, _p, _p, _p, _d, _p, _p, _i, _i, _i,
                                                    _i, _p]),
    "magmablas_dgemm_vbatched_max": (None, [_i, _i, _p, _p, _p, _d, _p, _p, _p, _p, _d, _p, _p, _i, _i, _i, _i, _p]),
    "magmablas_dgemm_vbatched_nocheck": (None, [_i, _i, _p, _p, _p, _d, _p, _p, _p, _p, _d, _p, _p, _i, _p]),
    "magmablas_sgemm_vbatched": (None, [_i, _i, _p, _p, _p, _f, _p, _p, _p, _p, _f, _p, _p, _i, _p]),
    "magmablas_sgemm_vbatched_max_nocheck": (None, [_i, _i, _p, _p, _p, _f, _p, _p, _p, _p, _f, _p, _p, _i, _i, _i,
                                                    _i, _p]),
    "magmablas_sgemm_vbatched_max": (None, [_i, _i, _p, _p, _p, _f, _p, _p, _p, _p, _f, _p, _p, _i, _i, _i, _i, _p]),
    "magmablas_sgemm_vbatched_nocheck": (None, [_i, _i, _p, _p, _p, _f, _p, _p, _p, _p, _f, _p, _p, _i, _p]),
    "magmablas_dsyrk_batched": (None, [_i, _i, _i, _i, _d, _p, _i, _d, _p, _i, _i, _p]),
    "magma_dsyrk_batched": (None, [_i, _i, _i, _i, _d, _p, _i, _d, _p, _i, _i, _p]),
    "magmablas_dtrsm_batched": (None, [_i, _i, _i, _i, _i, _i, _d, _p, _i, _p, _i, _i, _p]),
    "magmablas_dtrmm_batched": (None, [_i, _i, _i, _i, _i, _i, _d, _p, _i, _p, _i, _i, _p]),
    "magmablas_ssyrk_batched": (None, [_i, _i, _i, _i, _f, _p, _i, _f, _p, _i, _i, _p]),
    "magma_ssyrk_batched": (None, [_i, _i, _i, _i, _f, _p, _i, _f, _p, _i, _i, _p]),
    "magmablas_strsm_batched": (None, [_i, _i, _i, _i, _i, _i, _f, _p, _i, _p, _i, _i, _p]),
    "magmablas_strmm_batched": (None, [_i, _i, _i, _i, _i, _i, _f, _p, _i, _p, _i, _i, _p]),
    "magmablas_dsyrk_vbatched": (None, [_i, _i, _p, _p, _d, _p, _p, _d, _p, _p, _i, _p]),
    "magmablas_dsyrk_vbatched_max_nocheck": (None, [_i, _i, _p, _p, _d, _p, _p, _d, _p, _p, _i, _i, _i, _p]),
    "magmablas_dsyrk_vbatched_max": (None, [_i, _i, _p, _p, _d, _p, _p, _d, _p, _p, _i, _i, _i, _p]),
    "magmablas_dsyrk_vbatched_nocheck": (None, [_i, _i, _p, _p, _d, _p, _p, _d, _p, _p, _i, _p]),
    "magmablas_ssyrk_vbatched": (None, [_i, _i, _p, _p, _f, _p, _p, _f, _p, _p, _i, _p]),
    "magmablas_ssyrk_vbatched_max_nocheck": (None, [_i, _i, _p, _p, _f, _p, _p, _f, _p, _p, _i, _i, _i, _p]),
    "magmablas_ssyrk_vbatched_max": (None, [_i, _i, _p, _p, _f, _p, _p, _f, _p, _p, _i, _i, _i, _p]),
    "magmablas_ssyrk_vbatched_nocheck": (None, [_i, _i, _p, _p, _f, _p, _p, _f, _p, _p, _i, _p]),
    "magmablas_dtrsm_vbatched": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _p]),
    "magmablas_dtrsm_vbatched_max_nocheck": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_dtrsm_vbatched_max": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_dtrsm_vbatched_nocheck": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _p]),
    "magmablas_strsm_vbatched": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _p]),
    "magmablas_strsm_vbatched_max_nocheck": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_strsm_vbatched_max": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_strsm_vbatched_nocheck": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _p]),
    "magmablas_dtrmm_vbatched": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _p]),
    "magmablas_dtrmm_vbatched_max_nocheck": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_dtrmm_vbatched_max": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_dtrmm_vbatched_nocheck": (None, [_i, _i, _i, _i, _p, _p, _d, _p, _p, _p, _p, _i, _p]),
    "magmablas_strmm_vbatched": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _p]),
    "magmablas_strmm_vbatched_max_nocheck": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_strmm_vbatched_max": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _i, _i, _p]),
    "magmablas_strmm_vbatched_nocheck": (None, [_i, _i, _i, _i, _p, _p, _f, _p, _p, _p, _p, _i, _p]),
    "magma_dsposv_vbatched": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p]),
    "magma_dsposv_vbatched_max_nocheck": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p]),
    # kernel-variant tuning
    "magma_b200_autotune": (_i, [_p]),
    "magma_b200_tuning_get": (_i, [_p, _i]),
    "magma_b200_tuning_set": (_i, [_p, _i]),
    "magma_b200_tuning_save": (_i, [_s]),
    "magma_b200_tuning_load": (_i, [_s]),
    # request loop (include/magma_b200_serve.h)
    "magma_b200_host_solver_create": (_i, [_i, _i, _i, _i, _i, _i, _i, _p, C.POINTER(_p)]),
    "magma_b200_host_solve": (_i, [_p, _p, _p, _p, _p, _p]),
    "magma_b200_host_solver_chunk_start": (_i, [_p, _i]),
    "magma_b200_host_solver_destroy": (_i, [_p]),
    "magma_b200_server_create": (_i, [_i, _sz, _i, _i, C.POINTER(_p)]),
    "magma_b200_server_submit": (_i, [_p, _i, _i, _i, _p, _i, _p, _i, _p, _i, C.c_longlong]),
    "magma_b200_server_poll": (_i, [_p, _p, _p, _p, _p, _i]),
    "magma_b200_server_drain": (_i, [_p]),
    "magma_b200_server_set_workspace_limit": (_i, [_p, _sz]),
    "magma_b200_server_stats": (None, [_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "magma_b200_server_destroy": (_i, [_p]),
}

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load the library once and attach the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m magma_b200.build` "
            "(there is no CPU or library fallback)")
    # RTLD_LOCAL: the library exports MAGMA's C names; another MAGMA in the
    # process (torch bundles one in libtorch_cuda_linalg.so) must not resolve
    # its own calls to these definitions.
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
