"""GPU parity tests of the batched Cholesky path (fixed and variable size) through the C ABI.

The kernels apply the oracle's outer-product Cholesky operations (explicit
fma, multiplier = raw entry * (1/sqrt(d))) in the same order, so factors and
solutions must be BIT-IDENTICAL to the oracle; info must equal LAPACK's on
the golden vectors; factors agree with OpenBLAS dpotrf within
8*n*eps*sqrt(||A||_max)."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def spd_batch(batch, n, seed, lda=None):
    lda = lda or n
    A = np.zeros((batch, n, lda))
    for i in range(batch):
        A[i, :, :n] = T.spd_gram(n, seed, i)   # symmetric: column-major == row-major
    return A


def oracle_posv(A, B, upper=False, solve=True):
    batch, n, lda = A.shape
    As = [A[i] for i in range(batch)]
    Bs = [B[i] for i in range(batch)] if B is not None else [np.zeros((1, n)) for _ in range(batch)]
    nr = [B.shape[1] if B is not None else 1] * batch
    ldb = [B.shape[2] if B is not None else n] * batch
    return oracle.dposv_vbatched(As, Bs, [n] * batch, nr, [lda] * batch, ldb, solve=solve and B is not None,
                                 upper=upper)


@pytest.mark.parametrize("n", [1, 2, 5, 8, 16, 31, 32, 33, 64, 65, 100, 128, 200, 256, 300, 512, 700, 1024])
@pytest.mark.parametrize("upper", [False, True])
def test_potrf_bit_identical(cuda, n, upper):
    import magma_b200 as mb
    batch = max(2, min(64, 40000 // (n * n) + 2))
    A_np = spd_batch(batch, n, seed=n)
    A = dev(A_np, cuda)
    info = mb.dpotrf_batched(A, upper=upper)
    O = A_np.copy()
    oinf = oracle_posv(O, None, upper=upper, solve=False)
    assert np.array_equal(info.cpu().numpy(), oinf)
    G = A.cpu().numpy()
    tri = np.tril if not upper else np.triu
    for i in range(batch):   # only the referenced triangle is defined
        assert np.array_equal(tri(G[i].T), tri(O[i].T)), i
    # the other triangle is left untouched
    other = np.triu if not upper else np.tril
    assert np.array_equal(other(G[0].T, 1 if not upper else -1), other(A_np[0].T, 1 if not upper else -1))


@pytest.mark.parametrize("n,nrhs", [(4, 1), (16, 3), (32, 8), (48, 2), (64, 5), (100, 4), (256, 1), (400, 7)])
def test_posv_and_potrs_bit_identical(cuda, n, nrhs):
    import magma_b200 as mb
    batch = 24
    A_np = spd_batch(batch, n, seed=100 + n)
    B_np = T.normal(7, n, batch * nrhs * n).reshape(batch, nrhs, n)
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    info = mb.dposv_batched(A, B)
    OA, OB = A_np.copy(), B_np.copy()
    oinf = oracle_posv(OA, OB)
    assert np.array_equal(info.cpu().numpy(), oinf)
    assert np.array_equal(B.cpu().numpy(), OB)
    # potrs alone on the oracle's factors
    B2 = dev(B_np, cuda)
    mb.dpotrs_batched(dev(OA, cuda), B2)
    assert np.array_equal(B2.cpu().numpy(), OB)
    assert T.backward_error(A_np, OB, B_np, n).max() < 30 * EPS


def test_potrf_golden(cuda, chol_golden):
    import magma_b200 as mb
    g = chol_golden
    for tag in g["tags"]:
        a = g[f"{tag}/A"]
        n = a.shape[0]
        A = dev(np.ascontiguousarray(a.T)[None], cuda)
        info = mb.dpotrf_batched(A)
        assert info.item() == g[f"{tag}/info"], tag
        if info.item() == 0:
            L = np.tril(A.cpu().numpy()[0].T)
            assert np.abs(L - g[f"{tag}/L"]).max() <= 8 * n * EPS * np.sqrt(np.abs(a).max()), tag


def test_not_positive_definite(cuda):
    import magma_b200 as mb
    n = 40
    A_np = spd_batch(6, n, seed=3)
    A_np[1, 0, 0] = -1.0                     # first minor fails: info 1
    A_np[2, 17, 17] = -1e6                   # info 18
    A_np[3, 39, 39] = 0.0                    # last minor (likely positive anyway)
    A_np[4, 5, 5] = np.nan                   # NaN detected like LAPACK's DISNAN: info 6
    A = dev(A_np, cuda)
    info = mb.dpotrf_batched(A).cpu().numpy()
    oinf = oracle_posv(A_np.copy(), None, solve=False)
    assert np.array_equal(info, oinf)
    assert info[1] == 1 and info[2] == 18 and info[4] == 6 and info[0] == 0


def _power_law_sizes(count, lo, hi, seed):
    u = T.uniform01(seed, 11, count)
    # inverse CDF of p(n) ~ n^-1.5 on [lo, hi]
    a, b = lo ** -0.5, hi ** -0.5
    return np.clip(np.round((a - u * (a - b)) ** -2), lo, hi).astype(np.int32)


@pytest.mark.parametrize("checked", [True, False])
def test_posv_vbatched_bit_identical(cuda, checked):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    batch = 400
    ns = _power_law_sizes(batch, 1, 600, seed=5)
    ns[:3] = [1, 1024, 0]                    # extremes, including an empty instance
    nrhs = (1 + np.floor(T.uniform01(5, 12, batch) * 8)).astype(np.int32)
    lda = ((ns + 7) // 8) * 8
    lda[lda == 0] = 1
    As = [np.zeros((n, ld)) for n, ld in zip(ns, lda)]
    for i, n in enumerate(ns):
        if n:
            As[i][:, :n] = T.spd_gram(int(n), 9, i)
    Bs = [T.normal(9, 5000 + i, int(max(n, 1) * r)).reshape(r, max(n, 1)) for i, (n, r) in enumerate(zip(ns, nrhs))]
    ldb = [max(n, 1) for n in ns]
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    mx = None if checked else (int(ns.max()), int(nrhs.max()))
    info = mb.dposv_vbatched(gA, gB, ns, nrhs, lda, ldb, max_sizes=mx)
    OA = [a.copy() for a in As]
    OB = [b.copy() for b in Bs]
    oinf = oracle.dposv_vbatched(OA, OB, ns, nrhs, lda, ldb)
    assert np.array_equal(info.cpu().numpy(), oinf)
    RA, RB = gA.unpack(), gB.unpack()
    for i, n in enumerate(ns):
        assert np.array_equal(np.tril(RA[i][:, :n].T), np.tril(OA[i][:, :n].T)), (i, n)
        assert np.array_equal(RB[i], OB[i]), (i, n)


def test_potrf_vbatched_argument_errors(cuda):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    As = [np.eye(4), np.eye(3)]
    gA = VarBatch(As, cuda)
    with pytest.raises(ValueError, match="-2"):
        mb.dposv_vbatched(gA, None, [4, -1], lda=[4, 3], factor=True, solve=False)
    with pytest.raises(ValueError, match="-4"):
        mb.dposv_vbatched(gA, None, [4, 3], lda=[4, 2], factor=True, solve=False)
    info = mb.dposv_vbatched(gA, None, [4, 3], lda=[4, 3], factor=True, solve=False)
    assert info.cpu().tolist() == [0, 0]
