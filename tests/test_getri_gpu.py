"""GPU tests of the batched out-of-place inverse (magma_dgetri_outofplace_batched).

Each column of inv(A) is getrs applied to a unit vector, so the result is
BIT-IDENTICAL to the oracle's dgetrs with B = I; A inv(A) = I to rounding; info
reports the first exactly-zero U(i,i)."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("n,batch", [(1, 5), (3, 30), (8, 40), (17, 50), (31, 40), (32, 300), (33, 20), (63, 20),
                                     (100, 12), (256, 6), (520, 2)])
def test_getri_bit_identical(cuda, n, batch):
    import magma_b200 as mb
    A_np, _ = T.lu_uniform(batch, n, 1, seed=300 + n)
    A = dev(A_np, cuda)
    ipiv, info = mb.dgetrf_batched(A)
    inv, iinfo = mb.dgetri_outofplace_batched(A, ipiv)
    inv = inv.cpu().numpy()
    LU, ip = A.cpu().numpy(), ipiv.cpu().numpy()
    eye = np.tile(np.eye(n)[None], (batch, 1, 1))
    O = eye.copy()
    oracle.dgetrs_batched(LU.copy(), ip, O, trans=False)
    assert np.array_equal(inv, O)
    assert np.all(iinfo.cpu().numpy() == 0)
    for b in range(batch):
        Ar = A_np[b].T                      # row-major A
        X = inv[b].T
        assert np.abs(Ar @ X - np.eye(n)).max() <= 1e-9 * max(1.0, np.abs(X).max()) * n


@pytest.mark.parametrize("n", [20, 40])
def test_getri_reports_zero_pivot(cuda, n):
    import magma_b200 as mb
    A_np, _ = T.lu_uniform(3, n, 1, seed=9)
    A_np[1, 7, :] = 0.0                      # zero column 7 -> U(8,8) = 0
    A = dev(A_np, cuda)
    ipiv, info = mb.dgetrf_batched(A)
    _, iinfo = mb.dgetri_outofplace_batched(A, ipiv)
    assert list(iinfo.cpu().numpy()) == [0, int(info[1]), 0]
    assert int(info[1]) == 8


# ------------------------------------------------------------------ LU without pivoting
@pytest.mark.parametrize("n,nrhs,batch", [(1, 1, 5), (16, 2, 40), (32, 1, 40), (50, 3, 30), (64, 4, 20),
                                          (100, 2, 10), (256, 4, 6), (600, 1, 2)])
def test_gesv_nopiv_bit_identical(cuda, n, nrhs, batch):
    """Factors, info and solutions bit-identical to the oracle's dgetf2 without pivoting
    (diagonally dominant inputs keep the pivots away from zero)."""
    import magma_b200 as mb
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=700 + n)
    for i in range(n):
        A_np[:, i, i] += n                    # column-major: entry (i, i)
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    info = mb.dgesv_nopiv_batched(A, B)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_nopiv_batched(O, n)
    OB = B_np.copy()
    oracle.dgetrs_batched(O.copy(), oip, OB, trans=False)
    assert np.array_equal(info.cpu().numpy(), oinf)
    assert np.array_equal(A.cpu().numpy(), O)
    assert np.array_equal(B.cpu().numpy(), OB)
    assert T.backward_error(A_np, OB, B_np, n).max() < 30 * np.finfo(float).eps


@pytest.mark.parametrize("n", [24, 130])
def test_getrf_nopiv_zero_pivot_and_trans_solve(cuda, n):
    import magma_b200 as mb
    A_np, B_np = T.lu_uniform(3, n, 2, seed=41 + n)
    for i in range(n):
        A_np[:, i, i] += n
    A_np[1, 4, :] = 0.0                        # zero column 4: the step-5 pivot of instance 1 is exactly 0
    A = dev(A_np, cuda)
    info = mb.dgetrf_nopiv_batched(A)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_nopiv_batched(O, n)
    assert np.array_equal(info.cpu().numpy(), oinf) and oinf[1] == 5
    assert np.array_equal(np.nan_to_num(A.cpu().numpy()), np.nan_to_num(O))
    for trans in (False, True):
        Bd = dev(B_np[[0, 2]], cuda)
        mb.dgetrs_nopiv_batched(dev(O[[0, 2]], cuda), Bd, trans=trans)
        OB = B_np[[0, 2]].copy()
        oracle.dgetrs_batched(O[[0, 2]].copy(), oip[[0, 2]], OB, trans=trans)
        if not trans:
            assert np.array_equal(Bd.cpu().numpy(), OB)
        assert np.abs(Bd.cpu().numpy() - OB).max() <= 64 * n * np.finfo(float).eps * max(1.0, np.abs(OB).max())


# ------------------------------------------------------------------ random butterfly transformation
def _butterfly(n, w):
    """Dense depth-2 butterfly W = L2 L1 from its 2n weights (numpy, FP64)."""
    def level(order, ws):
        h = order // 2
        Bm = np.zeros((order, order))
        for i in range(h):
            Bm[i, i], Bm[i, h + i] = ws[i], ws[h + i]
            Bm[h + i, i], Bm[h + i, h + i] = ws[i], -ws[h + i]
        return Bm / np.sqrt(2.0)
    L1 = level(n, w[:n])
    L2 = np.zeros((n, n))
    L2[:n // 2, :n // 2] = level(n // 2, w[n:n + n // 2])
    L2[n // 2:, n // 2:] = level(n // 2, w[n + n // 2:])
    return L2 @ L1


@pytest.mark.parametrize("n", [8, 64, 100, 256])
def test_gerbt_matches_dense_transform(cuda, n):
    import magma_b200 as mb
    A_np, B_np = T.lu_uniform(4, n, 3, seed=60 + n)
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    u, v = mb.dgerbt_batched(A, B)
    Uw, Vw = _butterfly(n, u), _butterfly(n, v)
    for b in range(4):
        ref = Uw.T @ A_np[b].T @ Vw
        assert np.abs(A.cpu().numpy()[b].T - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
        rb = Uw.T @ B_np[b].T
        assert np.abs(B.cpu().numpy()[b].T - rb).max() <= 1e-13 * max(1.0, np.abs(rb).max())


@pytest.mark.parametrize("n", [16, 64, 128, 256])
def test_gesv_rbt_solves_without_pivoting(cuda, n):
    """RBT + LU without pivoting solves systems whose leading pivots are zero, where
    LU without pivoting alone breaks down."""
    import magma_b200 as mb
    batch, nrhs = 12, 2
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=90 + n)
    A_np[:, 0, 0] = 0.0                        # a zero first pivot: nopiv alone fails
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    info = mb.dgesv_rbt_batched(A, B)
    assert np.all(info.cpu().numpy() == 0)
    be = T.backward_error(A_np, B.cpu().numpy(), B_np, n)
    assert be.max() <= 1e-11, be.max()
    A2 = dev(A_np, cuda)
    info2 = mb.dgetrf_nopiv_batched(A2)
    assert np.all(info2.cpu().numpy() == 1)    # the untransformed system has pivot 1 == 0
