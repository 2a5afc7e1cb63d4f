"""CPU tests: the oracle restatement is pinned against the reference's LAPACK.

The golden vectors (tests/golden/*.npz, made by make_golden.py with scipy's
OpenBLAS, the LAPACK MAGMA's testers call) fix pivots and info exactly; the
factors and solutions of a different summation order must agree to
c*n*eps*||A||.
"""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

EPS = np.finfo(np.float64).eps


def _cm(a):
    """row-major (m, n) -> column-major storage (1, n, m)."""
    return np.ascontiguousarray(a.T)[None].copy()


def _tags(g, prefix=None):
    return [t for t in g["tags"] if prefix is None or t.startswith(prefix)]


def test_oracle_getrf_matches_lapack_golden(lu_golden):
    g = lu_golden
    for tag in _tags(g):
        m, n = (int(v) for v in g[f"{tag}/mn"])
        A = _cm(g[f"{tag}/A"])
        ipiv, info = oracle.dgetrf_batched(A, m)
        k = min(m, n)
        assert np.array_equal(ipiv[0, :k], g[f"{tag}/ipiv"][:k]), tag
        assert info[0] == g[f"{tag}/info"], tag
        if info[0] == 0:
            lu = A[0].T
            anorm = np.abs(g[f"{tag}/A"]).max()
            assert np.abs(lu - g[f"{tag}/LU"]).max() <= 8 * max(m, n) * EPS * max(anorm, 1.0), tag


def test_oracle_getrs_matches_lapack_golden(lu_golden):
    g = lu_golden
    for tag in _tags(g):
        if f"{tag}/B1" not in g:
            continue
        n = int(g[f"{tag}/mn"][0])
        LU = _cm(g[f"{tag}/LU"])
        ipiv = g[f"{tag}/ipiv"][None].astype(np.int32).copy()
        for nrhs in (1, 3):
            for trans, key in ((False, "XN"), (True, "XT")):
                B = np.ascontiguousarray(g[f"{tag}/B{nrhs}"].T)[None].copy()
                oracle.dgetrs_batched(LU, ipiv, B, trans=trans)
                X = g[f"{tag}/{key}{nrhs}"]
                scale = max(np.abs(X).max(), 1.0)
                assert np.abs(B[0].T - X).max() <= 64 * n * EPS * scale * 1e2, (tag, nrhs, trans)


def test_lapack_loop_is_the_golden_lapack(lu_golden):
    """The reference CPU loop (oracle.lapack_*) calls the same LAPACK as the fixtures: bit-identical."""
    g = lu_golden
    for tag in _tags(g, "uniform_32x32"):
        A = _cm(g[f"{tag}/A"])
        ipiv, info = oracle.lapack_dgetrf_batched(A, 32, nthreads=2)
        assert np.array_equal(A[0].T, g[f"{tag}/LU"])
        assert np.array_equal(ipiv[0], g[f"{tag}/ipiv"])


@pytest.mark.parametrize("n", [8, 32, 64])
def test_oracle_pivots_match_lapack_on_seeded_batch(n):
    """On the seeded U[-1,1] workload the restated getf2 and OpenBLAS pick identical pivots."""
    A, B = T.lu_uniform(1500, n, 2, seed=123 + n)
    A1, A2 = A.copy(), A.copy()
    B1, B2 = B.copy(), B.copy()
    ip1, inf1 = oracle.dgesv_batched(A1, B1)
    ip2, inf2 = oracle.lapack_dgesv_batched(A2, B2)
    assert np.array_equal(ip1, ip2)
    assert np.array_equal(inf1, inf2)
    assert np.abs(A1 - A2).max() < 64 * n * EPS
    be = T.backward_error(A, B1, B, n)
    assert be.max() < 30 * EPS


def test_oracle_singular_info():
    A = np.zeros((3, 8, 8))
    A[0] = np.eye(8)
    A[1] = np.eye(8)
    A[1, 5, :] = 0.0            # column 5 zero -> info 6
    ipiv, info = oracle.dgetrf_batched(A, 8)
    assert list(info) == [0, 6, 1]
    assert list(ipiv[2]) == list(range(1, 9))   # all-zero columns: no swaps, ipiv(k) = k


def test_generators_deterministic():
    a1 = T.uniform11(5, 0, 1000)
    a2 = T.uniform11(5, 0, 1000)
    assert np.array_equal(a1, a2)
    assert a1.min() >= -1 and a1.max() < 1
    assert abs(a1.mean()) < 0.1
    z = T.normal(5, 1, 20000)
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1) < 0.05
    M, N, K = T.gemm_sizes(5000)
    assert M.min() == 8 and M.max() == 128 and K.min() == 8 and N.max() == 128


def test_svd_logrand_condition():
    A, B, kap = T.svd_logrand(6, 48, 1e2, 1e6, nrhs=2, seed=9)
    for i in range(6):
        s = np.linalg.svd(A[i].T, compute_uv=False)
        assert s.max() <= 1 + 1e-12
        assert s.max() / s.min() <= kap[i] * (1 + 1e-8)
    assert kap.min() >= 1e2 and kap.max() <= 1e6


def test_oracle_cholesky_matches_lapack_golden(chol_golden):
    g = chol_golden
    for tag in g["tags"]:
        a = g[f"{tag}/A"]
        n = a.shape[0]
        A = [np.ascontiguousarray(a.T).copy()]
        has_b = f"{tag}/B" in g
        B = [np.ascontiguousarray(g[f"{tag}/B"].T).copy()] if has_b else [np.zeros((1, n))]
        info = oracle.dposv_vbatched(A, B, [n], [B[0].shape[0]], [n], [n], solve=has_b)
        assert info[0] == g[f"{tag}/info"], tag
        if info[0] == 0:
            L = np.tril(A[0].T)
            anorm = np.abs(a).max()
            assert np.abs(L - g[f"{tag}/L"]).max() <= 8 * n * EPS * np.sqrt(anorm), tag
            X = B[0].T
            assert np.abs(X - g[f"{tag}/X"]).max() <= 1e3 * n * EPS * max(np.abs(X).max(), 1), tag


def test_oracle_cholesky_upper_is_transpose():
    n = 23
    a = T.spd_gram(n, 5, 0)
    lo = [np.ascontiguousarray(a.T).copy()]
    up = [np.ascontiguousarray(a.T).copy()]
    b = np.ones((1, n))
    i1 = oracle.dposv_vbatched(lo, [b.copy()], [n], [1], [n], [n], solve=False)
    i2 = oracle.dposv_vbatched(up, [b.copy()], [n], [1], [n], [n], solve=False, upper=True)
    assert i1[0] == 0 and i2[0] == 0
    assert np.array_equal(np.tril(lo[0].T), np.triu(up[0].T).T)


@pytest.mark.parametrize("m,n", [(1, 1), (8, 8), (40, 17), (64, 64), (200, 50), (10, 30), (16, 33), (33, 40), (256, 64),
                                 (700, 20), (1024, 9)])
def test_oracle_geqr2_matches_lapack(m, n):
    """The restated dgeqr2 agrees with LAPACK dgeqrf (numpy's qr, mode 'raw') to rounding:
    same reflectors, same signs of R's diagonal, same tau."""
    rng = np.random.default_rng(m * 1000 + n)
    batch = 6
    A = rng.uniform(-1, 1, (batch, n, m))          # column-major (batch, n, lda=m)
    G = A.copy()
    tau = oracle.dgeqrf_batched(G, m)
    k = min(m, n)
    for b in range(batch):
        h, t = np.linalg.qr(A[b].T, mode="raw")    # h is LAPACK's column-major output
        assert np.abs(G[b] - h).max() < 64 * m * EPS
        assert np.abs(tau[b, :k] - t).max() < 64 * m * EPS


def test_oracle_geqr2_matches_reference_loop():
    """The restated dgeqr2 against the reference CPU loop (OpenBLAS dgeqrf per instance)."""
    m, n = 64, 64
    A, _ = T.lu_uniform(200, n, 1, seed=77)
    G1, G2 = A.copy(), A.copy()
    t1 = oracle.dgeqrf_batched(G1, m)
    t2 = oracle.lapack_dgeqrf_batched(G2, m, nthreads=2)
    assert np.abs(G1 - G2).max() < 64 * m * EPS
    assert np.abs(t1 - t2).max() < 64 * m * EPS


def test_reference_loop_getri_is_the_inverse():
    A, _ = T.lu_uniform(50, 24, 1, seed=5)
    X = A.copy()
    ipiv, info = oracle.lapack_dgetri_batched(X, nthreads=2)
    assert np.all(info == 0)
    for b in range(50):
        assert np.abs(A[b].T @ X[b].T - np.eye(24)).max() < 1e-10


def _tri_case(rng, solve, left, lower, trans, unit, m, n):
    k = m if left else n
    A = rng.uniform(-1, 1, (k, k + 3)) + np.eye(k, k + 3) * 4    # column-major (cols, lda)
    B = rng.uniform(-1, 1, (n, m + 2))
    return A, B


@pytest.mark.parametrize("solve", [True, False])
def test_oracle_tri_matches_blas(solve):
    """The restated trsm/trmm (the kernels' order) agrees with OpenBLAS dtrsm/dtrmm to
    rounding on all 16 side/uplo/trans/diag combinations."""
    rng = np.random.default_rng(11)
    for left in (True, False):
        for lower in (True, False):
            for trans in (True, False):
                for unit in (True, False):
                    m, n = 37, 21
                    A, B = _tri_case(rng, solve, left, lower, trans, unit, m, n)
                    B1, B2 = B.copy(), B.copy()
                    oracle.dtri(solve, left, lower, trans, unit, m, n, 0.75, A, B1)
                    oracle.lapack_dtri_vbatched(solve, left, lower, trans, unit, [m], [n], 0.75, [A], [A.shape[1]],
                                                [B2], [B2.shape[1]], nthreads=1)
                    scale = max(1.0, np.abs(B2).max())
                    assert np.abs(B1 - B2).max() < 64 * max(m, n) * EPS * scale, (left, lower, trans, unit)
                    assert np.array_equal(B1[:, m:], B[:, m:])      # padding rows untouched


def test_oracle_tri_alpha_zero():
    A = np.full((5, 5), np.nan)
    B = np.ones((4, 5))
    oracle.dtri(True, True, True, False, False, 5, 4, 0.0, A, B)
    assert np.all(B == 0.0)


@pytest.mark.parametrize("m,n", [(32, 32), (40, 24), (17, 30), (64, 64)])
def test_oracle_nopiv_is_the_pivoted_lu_when_the_diagonal_wins(m, n):
    """On column-wise diagonally dominant instances partial pivoting keeps every diagonal
    pivot, so the no-pivoting LU (the oracle of magma_dgetrf_nopiv_batched) must equal the
    pivoted getf2 restatement bit for bit -- that one is pinned to LAPACK on the golden
    vectors -- and LAPACK's own dgetrf to rounding, with LAPACK's identity pivots."""
    rng = np.random.default_rng(100 * m + n)
    batch, k = 20, min(m, n)
    A = rng.uniform(-1, 1, (batch, n, m))                   # column-major (batch, n, lda = m)
    for i in range(k):
        A[:, i, i] += max(m, n)
    P, Q, L = A.copy(), A.copy(), A.copy()
    ip_n, inf_n = oracle.dgetrf_nopiv_batched(P, m)
    ip_p, inf_p = oracle.dgetrf_batched(Q, m)
    ident = np.tile(np.arange(1, k + 1, dtype=np.int32), (batch, 1))
    assert np.array_equal(ip_p[:, :k], ident)                # no interchange happened
    assert np.array_equal(P, Q)
    assert not inf_n.any() and not inf_p.any()
    ip_l, inf_l = oracle.lapack_dgetrf_batched(L, m)
    assert np.array_equal(ip_l[:, :k], ident) and not inf_l.any()
    assert np.abs(P - L).max() <= 8 * max(m, n) * EPS * np.abs(A).max()
