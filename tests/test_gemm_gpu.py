"""GPU tests of the batched and variable-size GEMM through the C ABI.

Accuracy criterion of the reference's tester (testing_zgemm_vbatched.cpp:311-325):
||C - C_ref||_F / (sqrt(k+2) |alpha| ||A||_F ||B||_F + 2 |beta| ||C0||_F) < 30 eps,
with C_ref from float64 numpy (and the golden OpenBLAS dgemm/sgemm vectors)."""
import numpy as np
import pytest

from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def err(Cg, Cref, A, B, C0, k, alpha, beta):
    den = np.sqrt(k + 2) * abs(alpha) * np.linalg.norm(A) * np.linalg.norm(B) + 2 * abs(beta) * np.linalg.norm(C0)
    return np.linalg.norm(Cg - Cref) / max(den, 1e-300)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(8, 8, 8), (64, 64, 64), (65, 33, 17), (1, 70, 5), (128, 128, 128), (100, 31, 200)])
def test_gemm_batched(cuda, dt, ta, tb, m, n, k):
    import magma_b200 as mb
    batch, alpha, beta = 7, 0.29, -0.48
    eps = np.finfo(dt).eps
    Ar = T.normal(1, 1, batch * m * k).reshape(batch, m, k)
    Br = T.normal(1, 2, batch * k * n).reshape(batch, k, n)
    Cr = T.normal(1, 3, batch * m * n).reshape(batch, m, n)
    # column-major storage of op^{-1}: A stored as (cols, ld)
    A_st = (Ar.transpose(0, 2, 1) if not ta else Ar).astype(dt)     # (k, m) if not ta else (m, k) rows=cols
    B_st = (Br.transpose(0, 2, 1) if not tb else Br).astype(dt)
    C_st = Cr.transpose(0, 2, 1).astype(dt)
    Cg = dev(C_st, cuda)
    mb.gemm_batched(dev(A_st, cuda), dev(B_st, cuda), Cg, m, n, k, alpha, beta, ta, tb)
    got = Cg.cpu().numpy().transpose(0, 2, 1).astype(np.float64)
    a64, b64, c64 = Ar.astype(dt).astype(np.float64), Br.astype(dt).astype(np.float64), Cr.astype(dt).astype(np.float64)
    ref = alpha * a64 @ b64 + beta * c64
    for i in range(batch):
        assert err(got[i], ref[i], a64[i], b64[i], c64[i], k, alpha, beta) < 30 * eps, i


def test_gemm_beta_zero_ignores_c(cuda):
    import magma_b200 as mb
    m = n = k = 40
    A = T.normal(2, 1, m * k).reshape(1, k, m)
    B = T.normal(2, 2, k * n).reshape(1, n, k)
    C = np.full((1, n, m), np.nan)
    Cg = dev(C, cuda)
    mb.gemm_batched(dev(A, cuda), dev(B, cuda), Cg, m, n, k, 1.0, 0.0)
    assert np.isfinite(Cg.cpu().numpy()).all()


def test_gemm_golden(cuda, gemm_golden):
    import magma_b200 as mb
    g = gemm_golden
    for tag in g["tags"]:
        ta, tb = (bool(v) for v in g[f"{tag}/t"])
        a, b, c = g[f"{tag}/A"], g[f"{tag}/B"], g[f"{tag}/C"]
        m, n = c.shape
        k = a.shape[0] if ta else a.shape[1]
        for dt, key in ((np.float64, "D"), (np.float32, "S")):
            Cg = dev(c.T.astype(dt)[None], cuda)
            mb.gemm_batched(dev(a.T.astype(dt)[None], cuda), dev(b.T.astype(dt)[None], cuda), Cg, m, n, k, 1.0, 0.5,
                            ta, tb)
            got = Cg.cpu().numpy()[0].T.astype(np.float64)
            e = err(got, g[f"{tag}/{key}"].astype(np.float64), a, b, c, k, 1.0, 0.5)
            assert e < 30 * np.finfo(dt).eps, (tag, key, e)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("checked", [True, False])
def test_gemm_vbatched_config2(cuda, dt, checked):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    count = 2000
    M, N, K = T.gemm_sizes(count, 8, 128, seed=5)
    M[:2], N[:2], K[:2] = [1, 128], [128, 1], [1, 128]
    lda, ldb, ldc = T.roundup(M, 8), T.roundup(K, 8), T.roundup(M, 8)
    As = [np.zeros((k, l), dt) for k, l in zip(K, lda)]
    Bs = [np.zeros((n, l), dt) for n, l in zip(N, ldb)]
    Cs = [np.zeros((n, l), dt) for n, l in zip(N, ldc)]
    for i in range(count):
        As[i][:, :M[i]] = T.normal(7, 3 * i, M[i] * K[i]).reshape(K[i], M[i])
        Bs[i][:, :K[i]] = T.normal(7, 3 * i + 1, K[i] * N[i]).reshape(N[i], K[i])
        Cs[i][:, :M[i]] = T.normal(7, 3 * i + 2, M[i] * N[i]).reshape(N[i], M[i])
    tdt = torch.float64 if dt == np.float64 else torch.float32
    gA, gB, gC = VarBatch(As, cuda, tdt), VarBatch(Bs, cuda, tdt), VarBatch(Cs, cuda, tdt)
    alpha, beta = 1.0, 0.5
    mx = None if checked else (int(M.max()), int(N.max()), int(K.max()))
    mb.gemm_vbatched(gA, gB, gC, M, N, K, lda, ldb, ldc, alpha, beta, max_sizes=mx)
    out = gC.unpack()
    eps = np.finfo(dt).eps
    for i in range(count):
        a = As[i][:, :M[i]].T.astype(np.float64)
        b = Bs[i][:, :K[i]].T.astype(np.float64)
        c = Cs[i][:, :M[i]].T.astype(np.float64)
        ref = alpha * a @ b + beta * c
        got = out[i][:, :M[i]].T.astype(np.float64)
        assert err(got, ref, a, b, c, K[i], alpha, beta) < 30 * eps, i
        assert np.array_equal(out[i][:, M[i]:], Cs[i][:, M[i]:])   # padding rows untouched


def test_gemm_vbatched_argument_errors(cuda, capfd):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    A = VarBatch([np.eye(4)], cuda)
    mb.gemm_vbatched(A, A, A, [4], [4], [-1], [4], [4], [4])
    assert "parameter 5" in capfd.readouterr().err
    mb.gemm_vbatched(A, A, A, [4], [4], [4], [3], [4], [4])
    assert "parameter 8" in capfd.readouterr().err
    mb.gemm_vbatched(A, A, A, [4], [4], [4], [4], [4], [2])
    assert "parameter 13" in capfd.readouterr().err


@pytest.mark.parametrize("variant", ["max_nocheck", "max"])
def test_gemm_vbatched_max_argument_order(cuda, variant):
    """The _max_nocheck and _max forms take (..., lddc, batchCount, max_m, max_n, max_k, queue):
    the order of the reference's definitions (magmablas/zgemm_vbatched.cpp:19-29, 46-56)
    and of every call inside the reference (magmablas/ztrsm_vbatched_core.cu:235-236,
    zgemm_vbatched.cpp:99-106, testing/testing_zgemm_vbatched.cpp:244-251), which its
    public header declares as (max_m, max_n, max_k, batchCount). Called here with
    batchCount 5 and distinct maxima 16, 24, 40 over 40 allocated instances: the five
    products must be right and instances 5..39 untouched."""
    import ctypes as C

    import torch

    from magma_b200.api import VarBatch, default_queue
    q = default_queue()
    total, live = 40, 5
    M = np.full(total, 8, np.int32)
    N = np.full(total, 8, np.int32)
    K = np.full(total, 8, np.int32)
    M[:live], N[:live], K[:live] = [16, 3, 9, 16, 1], [24, 5, 24, 2, 7], [40, 11, 3, 40, 8]
    As = [T.normal(21, 3 * i, int(K[i] * M[i])).reshape(K[i], M[i]) for i in range(total)]
    Bs = [T.normal(21, 3 * i + 1, int(N[i] * K[i])).reshape(N[i], K[i]) for i in range(total)]
    Cs = [T.normal(21, 3 * i + 2, int(N[i] * M[i])).reshape(N[i], M[i]) for i in range(total)]
    gA, gB, gC = VarBatch(As, cuda), VarBatch(Bs, cuda), VarBatch(Cs, cuda)
    dm, dn, dk = gC.ints(M), gC.ints(N), gC.ints(K)
    vp = lambda t: C.c_void_p(t.data_ptr())
    fn = getattr(q.lib, f"magmablas_dgemm_vbatched_{variant}")
    fn(111, 111, vp(dm), vp(dn), vp(dk), 1.0, vp(gA.ptrs), vp(dm), vp(gB.ptrs), vp(dk), 0.5, vp(gC.ptrs), vp(dm),
       live, 16, 24, 40, q.handle)
    q.sync()
    out = gC.unpack()
    for i in range(total):
        if i < live:
            ref = As[i].T @ Bs[i].T + 0.5 * Cs[i].T
            assert err(out[i].T, ref, As[i], Bs[i], Cs[i], K[i], 1.0, 0.5) < 30 * np.finfo(np.float64).eps, i
        else:
            assert np.array_equal(out[i], Cs[i]), i
