"""GPU parity tests of the batched LU path through the C ABI.

The register-resident kernels perform LAPACK dgetf2 / reference-BLAS dtrsm
operations in the same order as the oracle restatement, so for them LU
factors, pivots, info and NoTrans solutions must be BIT-IDENTICAL to the
oracle; against the golden OpenBLAS outputs pivots and info must be identical
and factors within 8*max(m,n)*eps*||A||_max. Transposed solves use a
different (right-looking) order and are checked to 64*n*eps*||x||.
"""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def to_dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def gpu_getrf(A_np, m, dev):
    import magma_b200 as mb
    A = to_dev(A_np, dev)
    ipiv, info = mb.dgetrf_batched(A, m=m)
    return A.cpu().numpy(), ipiv.cpu().numpy(), info.cpu().numpy()


def test_getrf_golden_cases(cuda, lu_golden):
    g = lu_golden
    for tag in g["tags"]:
        m, n = (int(v) for v in g[f"{tag}/mn"])
        a = g[f"{tag}/A"]
        A_np = np.ascontiguousarray(a.T)[None].copy()
        LU, ipiv, info = gpu_getrf(A_np, m, cuda)
        # oracle: bit-identical
        O = A_np.copy()
        oip, oinf = oracle.dgetrf_batched(O, m)
        k = min(m, n)
        assert np.array_equal(ipiv[:, :k], oip[:, :k]), tag
        assert np.array_equal(info, oinf), tag
        assert np.array_equal(LU, O), tag
        # golden LAPACK: pivots/info identical, factors within tolerance
        assert np.array_equal(ipiv[0, :k], g[f"{tag}/ipiv"][:k]), tag
        assert info[0] == g[f"{tag}/info"], tag
        if info[0] == 0:
            assert np.abs(LU[0].T - g[f"{tag}/LU"]).max() <= 8 * max(m, n) * EPS * max(np.abs(a).max(), 1), tag


def test_getrs_golden_cases(cuda, lu_golden):
    import magma_b200 as mb
    g = lu_golden
    for tag in g["tags"]:
        if f"{tag}/B1" not in g:
            continue
        n = int(g[f"{tag}/mn"][0])
        LU = np.ascontiguousarray(g[f"{tag}/LU"].T)[None].copy()
        ip = g[f"{tag}/ipiv"][None].astype(np.int32).copy()
        for nrhs in (1, 3):
            for trans, key in ((False, "XN"), (True, "XT")):
                B_np = np.ascontiguousarray(g[f"{tag}/B{nrhs}"].T)[None].copy()
                Bd = to_dev(B_np, cuda)
                mb.dgetrs_batched(to_dev(LU, cuda), to_dev(ip, cuda), Bd, trans=trans)
                X = Bd.cpu().numpy()
                O = B_np.copy()
                oracle.dgetrs_batched(LU.copy(), ip, O, trans=trans)
                if not trans:
                    assert np.array_equal(X, O), (tag, nrhs)
                scale = max(np.abs(O).max(), 1.0)
                assert np.abs(X - O).max() <= 64 * n * EPS * scale, (tag, nrhs, trans)
                assert np.abs(X[0].T - g[f"{tag}/{key}{nrhs}"]).max() <= 1e4 * n * EPS * scale, (tag, nrhs, trans)


@pytest.mark.parametrize("n,nrhs", [(1, 1), (2, 1), (7, 2), (8, 1), (15, 5), (16, 4), (17, 1), (31, 1),
                                    (32, 1), (32, 4), (33, 3), (48, 1), (63, 9), (64, 1), (64, 16)])
def test_gesv_bit_identical(cuda, n, nrhs):
    import magma_b200 as mb
    batch = 777
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=1000 + n * 31 + nrhs)
    A = to_dev(A_np, cuda)
    B = to_dev(B_np, cuda)
    ipiv, info = mb.dgesv_batched(A, B)
    OA, OB = A_np.copy(), B_np.copy()
    oip, oinf = oracle.dgesv_batched(OA, OB)
    assert np.array_equal(ipiv.cpu().numpy(), oip)
    assert np.array_equal(info.cpu().numpy(), oinf)
    assert np.array_equal(A.cpu().numpy(), OA)
    assert np.array_equal(B.cpu().numpy(), OB)
    # the solution meets MAGMA's gesv check (testing_zgesv_batched.cpp:133-153)
    assert T.backward_error(A_np, OB, B_np, n).max() < 30 * EPS


@pytest.mark.parametrize("m,n", [(40, 24), (24, 40), (100, 64), (128, 20), (65, 65 - 1), (1, 9), (9, 1), (96, 33)])
def test_getrf_rectangular(cuda, m, n):
    batch = 301
    A_np, _ = T.lu_uniform(batch, n, 1, seed=77 + m + n, m=m)
    LU, ipiv, info = gpu_getrf(A_np, m, cuda)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_batched(O, m)
    assert np.array_equal(ipiv, oip)
    assert np.array_equal(info, oinf)
    assert np.array_equal(LU, O)
    assert T.lu_residual(A_np[:20], LU[:20], ipiv[:20], m, n).max() < 30 * EPS


def test_padded_leading_dimensions(cuda):
    import magma_b200 as mb
    n, nrhs = 29, 3
    A_np, B_np = T.lu_uniform(200, n, nrhs, seed=5, lda=40, ldb=37)
    A_np[:, :, n:] = 7.0     # padding must be left untouched
    B_np[:, :, n:] = -3.0
    A, B = to_dev(A_np, cuda), to_dev(B_np, cuda)
    ipiv, info = mb.dgesv_batched(A, B)
    OA, OB = A_np.copy(), B_np.copy()
    oracle.dgesv_batched(OA, OB)
    assert np.array_equal(A.cpu().numpy(), OA)
    assert np.array_equal(B.cpu().numpy(), OB)


def test_singular_instances(cuda):
    n = 16
    A_np, _ = T.lu_uniform(64, n, 1, seed=8)
    A_np[1, 5, :] = 0.0          # zero column 5 -> info 6
    A_np[2] = 0.0                # zero matrix -> info 1
    A_np[3, :, 0] = 0.0          # zero row 0 -> rank deficient
    A_np[3, :, 1] = A_np[3, :, 2]
    LU, ipiv, info = gpu_getrf(A_np, n, cuda)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_batched(O, n)
    assert info[1] == 6 and info[2] == 1
    assert np.array_equal(info, oinf)
    assert np.array_equal(ipiv, oip)
    assert np.array_equal(np.nan_to_num(LU), np.nan_to_num(O))


def test_config1_full_size(cuda):
    """10,000 x (32x32) U[-1,1], 1 RHS: pivots, info, LU and x bit-identical to the oracle
    and pivots identical to the reference CPU LAPACK loop."""
    import magma_b200 as mb
    A_np, B_np = T.lu_uniform(10000, 32, 1, seed=1)
    A, B = to_dev(A_np, cuda), to_dev(B_np, cuda)
    ipiv, info = mb.dgesv_batched(A, B)
    OA, OB = A_np.copy(), B_np.copy()
    oip, oinf = oracle.dgesv_batched(OA, OB)
    LA, LB = A_np.copy(), B_np.copy()
    lip, linf = oracle.lapack_dgesv_batched(LA, LB)
    g_ip, g_inf = ipiv.cpu().numpy(), info.cpu().numpy()
    assert np.array_equal(g_ip, oip) and np.array_equal(g_inf, oinf)
    assert np.array_equal(g_ip, lip) and np.array_equal(g_inf, linf)
    assert np.array_equal(A.cpu().numpy(), OA)
    assert np.array_equal(B.cpu().numpy(), OB)
    be = T.backward_error(A_np, B.cpu().numpy(), B_np, 32)
    assert be.max() <= 1e-14


# ------------------------------------------------------------------ blocked path (n > 64)
@pytest.mark.parametrize("n,nrhs,batch", [(65, 1, 64), (96, 3, 64), (100, 4, 48), (128, 1, 48), (129, 5, 32),
                                          (200, 2, 24), (256, 4, 32), (300, 1, 12), (512, 4, 6), (700, 2, 3),
                                          (1024, 1, 2)])
def test_blocked_gesv_bit_identical(cuda, n, nrhs, batch):
    import magma_b200 as mb
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=4000 + n + nrhs)
    A, B = to_dev(A_np, cuda), to_dev(B_np, cuda)
    ipiv, info = mb.dgesv_batched(A, B)
    OA, OB = A_np.copy(), B_np.copy()
    oip, oinf = oracle.dgesv_batched(OA, OB)
    assert np.array_equal(ipiv.cpu().numpy(), oip)
    assert np.array_equal(info.cpu().numpy(), oinf)
    assert np.array_equal(A.cpu().numpy(), OA)
    assert np.array_equal(B.cpu().numpy(), OB)
    assert T.backward_error(A_np, OB, B_np, n).max() < 30 * EPS


@pytest.mark.parametrize("m,n", [(200, 80), (80, 200), (256, 255), (500, 33), (129, 1000), (1024, 64)])
def test_blocked_getrf_rectangular(cuda, m, n):
    batch = 5
    A_np, _ = T.lu_uniform(batch, n, 1, seed=55 + m + n, m=m)
    LU, ipiv, info = gpu_getrf(A_np, m, cuda)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_batched(O, m)
    assert np.array_equal(ipiv, oip)
    assert np.array_equal(info, oinf)
    assert np.array_equal(LU, O)


@pytest.mark.parametrize("n", [90, 256, 333])
def test_blocked_getrs_trans(cuda, n):
    import magma_b200 as mb
    batch, nrhs = 6, 3
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=99 + n)
    O = A_np.copy()
    oip, _ = oracle.dgetrf_batched(O, n)
    for trans in (False, True):
        Bd = to_dev(B_np, cuda)
        mb.dgetrs_batched(to_dev(O, cuda), to_dev(oip, cuda), Bd, trans=trans)
        X = Bd.cpu().numpy()
        OB = B_np.copy()
        oracle.dgetrs_batched(O.copy(), oip, OB, trans=trans)
        if not trans:
            assert np.array_equal(X, OB)
        assert np.abs(X - OB).max() <= 64 * n * EPS * max(np.abs(OB).max(), 1.0)


def test_blocked_singular(cuda):
    n = 150
    A_np, _ = T.lu_uniform(4, n, 1, seed=3)
    A_np[1, 77, :] = 0.0   # zero column 77 -> info 78
    A_np[2] = 0.0
    LU, ipiv, info = gpu_getrf(A_np, n, cuda)
    O = A_np.copy()
    oip, oinf = oracle.dgetrf_batched(O, n)
    assert info[1] == 78 and info[2] == 1
    assert np.array_equal(info, oinf) and np.array_equal(ipiv, oip)
    assert np.array_equal(np.nan_to_num(LU), np.nan_to_num(O))


@pytest.mark.parametrize("n,nrhs,batch,chunks", [(32, 1, 1001, 4), (20, 3, 5, 8), (100, 2, 33, 3)])
def test_gesv_host_pipelined_matches_oracle(cuda, n, nrhs, batch, chunks):
    """HostDgesv (pinned host buffers, uploads/solves/read-backs overlapped chunk by chunk)
    returns the oracle's X, ipiv and info bit for bit; one instance is singular."""
    import torch
    from magma_b200.api import HostDgesv, default_queue
    A_np, B_np = T.lu_uniform(batch, n, nrhs, seed=5 * n + batch)
    A_np[2, 4, :] = 0.0                                      # column 5 zero -> info = 5
    OA, OB = A_np.copy(), B_np.copy()
    oip, oinf = oracle.dgesv_batched(OA, OB)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hA, hB = pin(A_np), pin(B_np)
    hX = torch.full(B_np.shape, np.nan, dtype=torch.float64).pin_memory()
    hP = torch.zeros((batch, n), dtype=torch.int32).pin_memory()
    hI = torch.full((batch,), 99, dtype=torch.int32).pin_memory()
    solver = HostDgesv(batch, n, nrhs, chunks=chunks)
    for _ in range(2):                                       # the staging buffers are reused
        hX.fill_(np.nan)
        solver(hA, hB, hX, hP, hI)
        default_queue().stream.synchronize()
        assert np.array_equal(hP.numpy(), oip)
        assert np.array_equal(hI.numpy(), oinf) and oinf[2] == 5
        ok = oinf == 0
        assert np.array_equal(hX.numpy()[ok], OB[ok])
    with pytest.raises(ValueError):
        solver(hA, hB, hX, hP[:, :1].clone().pin_memory(), hI)   # wrong output shape
