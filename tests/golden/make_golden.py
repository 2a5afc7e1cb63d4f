"""Generate the golden vectors that pin the oracle to the reference's CPU LAPACK.

The reference (MAGMA 2.2) ships no golden vectors for its batched path; its
testers compare against host LAPACK at run time (testing_zgetrf_batched.cpp:200,
testing_zgesv_batched.cpp:171, testing_zpotrf_vbatched.cpp:166,
testing_zgemm_vbatched.cpp:293). This script runs that LAPACK -- OpenBLAS
0.3.30 as bundled with scipy 1.18.1 -- through scipy.linalg.lapack on seeded
inputs from magma_b200.testing and stores inputs and outputs:

  lu_golden.npz      dgetrf / dgetrs (N and T) / dgesv: LU, ipiv (1-based), info, X
  chol_golden.npz    dpotrf / dpotrs: L, info, X (SPD and non-SPD instances)
  gemm_golden.npz    dgemm / sgemm on varied shapes

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
import zlib
from pathlib import Path

import numpy as np
import scipy
import scipy.linalg.lapack as lapack
import scipy.linalg.blas as blas

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from magma_b200 import testing as T  # noqa: E402

OUT = Path(__file__).resolve().parent


def lu_cases():
    """(tag, m, n, A row-major) for the LU fixtures."""
    cases = []
    sizes = [(1, 1), (2, 2), (3, 3), (5, 5), (8, 8), (13, 13), (16, 16), (31, 31), (32, 32),
             (33, 33), (47, 47), (64, 64), (40, 24), (24, 40), (100, 64), (1, 7), (7, 1)]
    seed = 11
    for (m, n) in sizes:
        for r in range(4):
            a = T.uniform11(seed, 0, m * n).reshape(n, m).T.copy()
            cases.append((f"uniform_{m}x{n}_{r}", m, n, a))
            seed += 1
    # first-step exact ties: |x| equal in several rows of column 0
    for n in (4, 9, 32, 64):
        for r in range(3):
            a = T.uniform11(seed, 0, n * n).reshape(n, n).T.copy()
            col = np.where(T.uniform01(seed, 3, n) < 0.5, -1.0, 1.0) * 2.0
            a[:, 0] = col
            cases.append((f"tie_{n}_{r}", n, n, a))
            seed += 1
    # structurally singular: a zero column at j -> info = j+1
    for n, j in ((5, 0), (8, 3), (32, 31), (33, 17), (64, 40)):
        a = T.uniform11(seed, 0, n * n).reshape(n, n).T.copy()
        a[:, j] = 0.0
        cases.append((f"zerocol_{n}_{j}", n, n, a))
        seed += 1
    cases.append(("zeros_6", 6, 6, np.zeros((6, 6))))
    # rank-one: info > 0 after the first step (exact zeros appear only if exact)
    v = np.arange(1.0, 9.0)
    cases.append(("rank1_8", 8, 8, np.outer(v, v[::-1])))
    return cases


def make_lu():
    out = {}
    tags = []
    for tag, m, n, a in lu_cases():
        lu, piv, info = lapack.dgetrf(a.copy())
        out[f"{tag}/A"] = a
        out[f"{tag}/LU"] = lu
        out[f"{tag}/ipiv"] = (piv + 1).astype(np.int32)
        out[f"{tag}/info"] = np.int32(info)
        out[f"{tag}/mn"] = np.array([m, n], np.int32)
        if m == n and info == 0:
            for nrhs in (1, 3):
                b = T.uniform11(zlib.crc32(tag.encode()) % 100000 + nrhs, 1, n * nrhs).reshape(nrhs, n).T.copy()
                xn, _ = lapack.dgetrs(lu, piv, b.copy(), trans=0)
                xt, _ = lapack.dgetrs(lu, piv, b.copy(), trans=1)
                out[f"{tag}/B{nrhs}"] = b
                out[f"{tag}/XN{nrhs}"] = xn
                out[f"{tag}/XT{nrhs}"] = xt
        tags.append(tag)
    out["tags"] = np.array(tags)
    out["lapack"] = np.array([f"scipy {scipy.__version__} / OpenBLAS (scipy_openblas)"])
    np.savez_compressed(OUT / "lu_golden.npz", **out)
    print("lu_golden.npz:", len(tags), "cases")


def make_chol():
    out = {}
    tags = []
    for i, n in enumerate((1, 2, 4, 7, 8, 16, 31, 32, 33, 48, 64, 65, 100, 128)):
        a = T.spd_gram(n, 21, i)
        l, info = lapack.dpotrf(a.copy(), lower=1, clean=1)
        b = T.normal(21, 50 + i, n * 3).reshape(3, n).T.copy()
        x, info2 = lapack.dpotrs(l, b.copy(), lower=1)
        tag = f"spd_{n}"
        out[f"{tag}/A"], out[f"{tag}/L"], out[f"{tag}/info"] = a, l, np.int32(info)
        out[f"{tag}/B"], out[f"{tag}/X"] = b, x
        tags.append(tag)
    # not positive definite: make the k-th leading minor fail
    for i, (n, k) in enumerate(((5, 1), (8, 4), (32, 20), (64, 64))):
        a = T.spd_gram(n, 22, i)
        a[k - 1, k - 1] = -abs(a[k - 1, k - 1]) - 1e3 * n
        l, info = lapack.dpotrf(a.copy(), lower=1, clean=0)
        tag = f"nonspd_{n}_{k}"
        out[f"{tag}/A"], out[f"{tag}/info"] = a, np.int32(info)
        tags.append(tag)
    out["tags"] = np.array(tags)
    np.savez_compressed(OUT / "chol_golden.npz", **out)
    print("chol_golden.npz:", len(tags), "cases")


def make_gemm():
    out = {}
    tags = []
    shapes = [(8, 8, 8), (17, 9, 33), (64, 48, 40), (1, 64, 5), (64, 1, 7), (45, 77, 1), (100, 31, 24)]
    for i, (m, n, k) in enumerate(shapes):
        for ta, tb in ((0, 0), (1, 0), (0, 1), (1, 1)):
            a = T.normal(31, 3 * i, m * k).reshape((k, m) if ta else (m, k))
            b = T.normal(31, 3 * i + 1, k * n).reshape((n, k) if tb else (k, n))
            c = T.normal(31, 3 * i + 2, m * n).reshape(m, n)
            tag = f"g{m}x{n}x{k}_{ta}{tb}"
            out[f"{tag}/A"], out[f"{tag}/B"], out[f"{tag}/C"] = a, b, c
            out[f"{tag}/D"] = blas.dgemm(1.0, a, b, 0.5, c.copy(), trans_a=ta, trans_b=tb)
            out[f"{tag}/S"] = blas.sgemm(1.0, a.astype(np.float32), b.astype(np.float32), 0.5,
                                         c.astype(np.float32), trans_a=ta, trans_b=tb)
            out[f"{tag}/t"] = np.array([ta, tb], np.int32)
            tags.append(tag)
    out["tags"] = np.array(tags)
    np.savez_compressed(OUT / "gemm_golden.npz", **out)
    print("gemm_golden.npz:", len(tags), "cases")


if __name__ == "__main__":
    make_lu()
    make_chol()
    make_gemm()
