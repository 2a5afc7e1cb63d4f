"""CPU oracle for the batched dense path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package. It wraps liboracle.so (built from oracle/*.c by oracle/Makefile):

* ``dgetrf_batched`` / ``dgetrs_batched`` / ``dgesv_batched``: the project's
  restatement of LAPACK dgetf2/dgetrs (see lapack_oracle.c for the exact
  operation order, which the GPU kernels reproduce bit for bit);
* ``lapack_*``: the reference's CPU path itself -- an OpenMP loop calling the
  image's LAPACK (OpenBLAS 0.3.30 from scipy) once per instance, as MAGMA's
  testers do (testing/testing_zgetrf_batched.cpp:188-206).

Matrices are column-major: an (m x n) instance with leading dimension ld is
stored as a numpy array of shape (n, ld) (row j = column j), and a batch as
shape (batch, n, ld).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_lib = None
_lapack_ready = False

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def build() -> Path:
    """Compile liboracle.so (make -C oracle)."""
    r = subprocess.run(["make", "-C", str(_HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return _LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(_LIB_PATH))
    return _lib


def openblas_path() -> str:
    import scipy

    cands = sorted(glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                          "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy-bundled OpenBLAS not found")
    return os.path.realpath(cands[0])


def _lapack() -> C.CDLL:
    global _lapack_ready
    L = lib()
    if not _lapack_ready:
        if L.lapack_loop_init(openblas_path().encode()) != 0:
            raise RuntimeError("could not load LAPACK symbols from scipy's OpenBLAS")
        _lapack_ready = True
    return L


def max_threads() -> int:
    return int(lib().lapack_loop_max_threads())


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _f(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def _ptrs(arrs, ctype):
    return (C.POINTER(ctype) * len(arrs))(*[a.ctypes.data_as(C.POINTER(ctype)) for a in arrs])


# ---------------------------------------------------------------- restatement
def dgetrf_batched(A: np.ndarray, m: int):
    """In-place LU of a (batch, n, lda) column-major batch. Returns (ipiv, info)."""
    batch, n, lda = A.shape
    ipiv = np.zeros((batch, max(1, min(m, n))), np.int32)
    info = np.zeros(batch, np.int32)
    lib().oracle_dgetrf_batched(m, n, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(ipiv.shape[1]),
                                _i(info), batch)
    return ipiv, info


def dgetrf_nopiv_batched(A: np.ndarray, m: int):
    """In-place LU without pivoting. Returns (ipiv = identity sequence, info)."""
    batch, n, lda = A.shape
    ipiv = np.zeros((batch, max(1, min(m, n))), np.int32)
    info = np.zeros(batch, np.int32)
    lib().oracle_dgetrf_nopiv_batched(m, n, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(ipiv.shape[1]),
                                      _i(info), batch)
    return ipiv, info


def dgeqrf_batched(A: np.ndarray, m: int):
    """In-place Householder QR (dgeqr2 restatement) of a (batch, n, lda) batch. Returns tau."""
    batch, n, lda = A.shape
    tau = np.zeros((batch, max(1, min(m, n))))
    lib().oracle_dgeqrf_batched(m, n, _d(A), lda, C.c_long(n * lda), _d(tau), C.c_long(tau.shape[1]), batch)
    return tau


def dtri(solve: bool, left: bool, lower: bool, trans: bool, unit: bool, m: int, n: int, alpha: float,
         A: np.ndarray, B: np.ndarray):
    """trsm (solve) / trmm in the batched kernels' order, in place on one column-major
    instance: A is (k, lda) with k = m (left) or n (right), B is (n, ldb)."""
    lib().oracle_dtri(int(solve), int(left), int(lower), int(trans), int(unit), m, n, C.c_double(alpha), _d(A),
                      A.shape[1], _d(B), B.shape[1])


def dgetrs_batched(A: np.ndarray, ipiv: np.ndarray, B: np.ndarray, trans: bool = False):
    """Solve with the factors; B is (batch, nrhs, ldb), overwritten with X."""
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    lib().oracle_dgetrs_batched(int(trans), n, nrhs, _d(A), lda, C.c_long(n * lda), _i(ipiv),
                                C.c_long(ipiv.shape[1]), _d(B), ldb, C.c_long(nrhs * ldb), batch)


def dgesv_batched(A: np.ndarray, B: np.ndarray):
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    ipiv = np.zeros((batch, n), np.int32)
    info = np.zeros(batch, np.int32)
    lib().oracle_dgesv_batched(n, nrhs, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(n), _d(B), ldb,
                               C.c_long(nrhs * ldb), _i(info), batch)
    return ipiv, info


def dposv_vbatched(As, Bs, ns, nrhss, ldas, ldbs, solve=True, upper=False):
    """Restated Cholesky (+ solve) on lists of column-major arrays, in place. Returns info."""
    batch = len(As)
    info = np.zeros(batch, np.int32)
    n, nr, la, lb = (np.asarray(v, np.int32) for v in (ns, nrhss, ldas, ldbs))
    Bl = Bs if Bs is not None else As
    lib().oracle_dposv_vbatched(int(upper), _i(n), _i(nr), _ptrs(As, C.c_double), _i(la),
                                _ptrs(Bl, C.c_double), _i(lb), _i(info), batch, int(solve))
    return info


# ---------------------------------------------------- reference CPU LAPACK loop
def lapack_dgetrf_batched(A: np.ndarray, m: int, nthreads: int | None = None):
    batch, n, lda = A.shape
    ipiv = np.zeros((batch, max(1, min(m, n))), np.int32)
    info = np.zeros(batch, np.int32)
    _lapack().ref_dgetrf_batched(m, n, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(ipiv.shape[1]),
                                 _i(info), batch, nthreads or max_threads())
    return ipiv, info


def lapack_dgetrs_batched(A, ipiv, B, trans=False, nthreads=None):
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    _lapack().ref_dgetrs_batched(int(trans), n, nrhs, _d(A), lda, C.c_long(n * lda), _i(ipiv),
                                 C.c_long(ipiv.shape[1]), _d(B), ldb, C.c_long(nrhs * ldb), batch,
                                 nthreads or max_threads())


def lapack_dgesv_batched(A: np.ndarray, B: np.ndarray, nthreads: int | None = None):
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    ipiv = np.zeros((batch, n), np.int32)
    info = np.zeros(batch, np.int32)
    _lapack().ref_dgesv_batched(n, nrhs, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(n), _d(B), ldb,
                                C.c_long(nrhs * ldb), _i(info), batch, nthreads or max_threads())
    return ipiv, info


def lapack_dgeqrf_batched(A: np.ndarray, m: int, nthreads: int | None = None):
    """LAPACK dgeqrf per instance, in place on a (batch, n, lda) batch; returns tau."""
    batch, n, lda = A.shape
    tau = np.zeros((batch, max(1, min(m, n))))
    _lapack().ref_dgeqrf_batched(m, n, _d(A), lda, C.c_long(n * lda), _d(tau), C.c_long(tau.shape[1]), batch,
                                 nthreads or max_threads())
    return tau


def lapack_dgetri_batched(A: np.ndarray, nthreads: int | None = None):
    """LAPACK dgetrf + dgetri per instance, in place (A becomes inv(A)); returns (ipiv, info)."""
    batch, n, lda = A.shape
    ipiv = np.zeros((batch, n), np.int32)
    info = np.zeros(batch, np.int32)
    _lapack().ref_dgetri_batched(n, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(n), _i(info), batch,
                                 nthreads or max_threads())
    return ipiv, info


def lapack_dsgesv_batched(A: np.ndarray, B: np.ndarray, nthreads: int | None = None):
    """LAPACK dsgesv per instance; returns (X, ipiv, iter, info)."""
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    X = np.zeros((batch, nrhs, n), np.float64)
    ipiv = np.zeros((batch, n), np.int32)
    it = np.zeros(batch, np.int32)
    info = np.zeros(batch, np.int32)
    _lapack().ref_dsgesv_batched(n, nrhs, _d(A), lda, C.c_long(n * lda), _i(ipiv), C.c_long(n), _d(B), ldb,
                                 C.c_long(nrhs * ldb), _d(X), n, C.c_long(nrhs * n), _i(it), _i(info), batch,
                                 nthreads or max_threads())
    return X, ipiv, it, info


def lapack_dposv_vbatched(As, Bs, ns, nrhss, ldas, ldbs, solve=True, nthreads=None):
    """Per-instance dpotrf (+dpotrs) on lists of column-major arrays (in place)."""
    batch = len(As)
    info = np.zeros(batch, np.int32)
    n = np.asarray(ns, np.int32)
    nr = np.asarray(nrhss, np.int32)
    la = np.asarray(ldas, np.int32)
    lb = np.asarray(ldbs, np.int32)
    _lapack().ref_dposv_vbatched(_i(n), _i(nr), _ptrs(As, C.c_double), _i(la), _ptrs(Bs, C.c_double), _i(lb),
                                 _i(info), batch, int(solve), nthreads or max_threads())
    return info


def lapack_gemm_vbatched(ta, tb, ms, ns, ks, alpha, As, ldas, Bs, ldbs, beta, Cs, ldcs, nthreads=None):
    batch = len(As)
    dt = As[0].dtype
    m, n, k, la, lb, lc = (np.asarray(v, np.int32) for v in (ms, ns, ks, ldas, ldbs, ldcs))
    if dt == np.float64:
        _lapack().ref_dgemm_vbatched(int(ta), int(tb), _i(m), _i(n), _i(k), C.c_double(alpha),
                                     _ptrs(As, C.c_double), _i(la), _ptrs(Bs, C.c_double), _i(lb),
                                     C.c_double(beta), _ptrs(Cs, C.c_double), _i(lc), batch,
                                     nthreads or max_threads())
    else:
        _lapack().ref_sgemm_vbatched(int(ta), int(tb), _i(m), _i(n), _i(k), C.c_float(alpha),
                                     _ptrs(As, C.c_float), _i(la), _ptrs(Bs, C.c_float), _i(lb),
                                     C.c_float(beta), _ptrs(Cs, C.c_float), _i(lc), batch,
                                     nthreads or max_threads())


def lapack_dtri_vbatched(solve, left, lower, trans, unit, ms, ns, alpha, As, ldas, Bs, ldbs, nthreads=None):
    """BLAS dtrsm (solve) / dtrmm per instance, in place on lists of column-major arrays."""
    batch = len(Bs)
    _lapack().ref_dtri_vbatched(int(solve), int(left), int(lower), int(trans), int(unit),
                                _i(np.asarray(ms, np.int32)), _i(np.asarray(ns, np.int32)), C.c_double(alpha),
                                _ptrs(As, C.c_double), _i(np.asarray(ldas, np.int32)), _ptrs(Bs, C.c_double),
                                _i(np.asarray(ldbs, np.int32)), batch, nthreads or max_threads())


def lapack_dsyrk_vbatched(lower, trans, ns, ks, alpha, As, ldas, beta, Cs, ldcs, nthreads=None):
    """BLAS dsyrk per instance, in place on lists of column-major arrays."""
    batch = len(Cs)
    _lapack().ref_dsyrk_vbatched(int(lower), int(trans), _i(np.asarray(ns, np.int32)), _i(np.asarray(ks, np.int32)),
                                 C.c_double(alpha), _ptrs(As, C.c_double), _i(np.asarray(ldas, np.int32)),
                                 C.c_double(beta), _ptrs(Cs, C.c_double), _i(np.asarray(ldcs, np.int32)), batch,
                                 nthreads or max_threads())
