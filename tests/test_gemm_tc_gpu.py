"""GPU tests of the FP32 GEMM tile on the tcgen05 tensor cores (FP32 tuning variant 3:
split TF32, FP32 accumulation in tensor memory), through the C ABI.

The tile is not bit-identical to the CUDA-core FP32 tiles, so it is held to the
reference tester's criterion (testing_zgemm_vbatched.cpp:311-325):
||C - C_ref||_F / (sqrt(k+2) |alpha| ||A||_F ||B||_F + 2 |beta| ||C0||_F) < 30 eps,
with C_ref from float64 numpy: every transpose form, sizes across one and several
128x128 tiles, K not a multiple of the 32-wide chunk (and K = 0: the reference's quick
return, C untouched), beta = 0 (C not read),
variable sizes and the SYRK triangle masks."""
import ctypes as C

import numpy as np
import pytest

from magma_b200 import _lib
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def err(Cg, Cref, A, B, C0, k, alpha, beta):
    den = np.sqrt(k + 2) * abs(alpha) * np.linalg.norm(A) * np.linalg.norm(B) + 2 * abs(beta) * np.linalg.norm(C0)
    return np.linalg.norm(Cg - Cref) / max(den, 1e-300)


@pytest.fixture
def fp32_tensor_core_tile():
    lib = _lib.load()
    count = lib.magma_b200_tuning_get(None, 0)
    vals = (C.c_int * count)()
    assert lib.magma_b200_tuning_get(vals, count) == count
    old = list(vals)
    for b in range(4):
        vals[4 + b] = 3            # FP32 GEMM tile of every size bucket
    assert lib.magma_b200_tuning_set(vals, count) == 0
    yield
    assert lib.magma_b200_tuning_set((C.c_int * count)(*old), count) == 0


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(8, 8, 8), (64, 64, 64), (65, 33, 17), (1, 70, 5), (128, 128, 128),
                                   (100, 31, 200), (200, 150, 70), (129, 257, 33), (17, 5, 0)])
def test_gemm_batched_fp32_tensor_core(cuda, fp32_tensor_core_tile, ta, tb, m, n, k):
    import magma_b200 as mb
    batch, alpha, beta = 5, 0.29, -0.48
    eps = np.finfo(np.float32).eps
    Ar = T.normal(3, 1, batch * m * k).reshape(batch, m, k)
    Br = T.normal(3, 2, batch * k * n).reshape(batch, k, n)
    Cr = T.normal(3, 3, batch * m * n).reshape(batch, m, n)
    A_st = (Ar.transpose(0, 2, 1) if not ta else Ar).astype(np.float32)
    B_st = (Br.transpose(0, 2, 1) if not tb else Br).astype(np.float32)
    C_st = Cr.transpose(0, 2, 1).astype(np.float32)
    if k == 0:   # keep a non-empty leading dimension for the empty operands
        A_st = np.zeros((batch, 1, m if not ta else 1), np.float32) if not ta else np.zeros((batch, m, 1), np.float32)
        B_st = np.zeros((batch, n, 1), np.float32) if not tb else np.zeros((batch, 1, n), np.float32)
    Cg = dev(C_st, cuda)
    mb.gemm_batched(dev(A_st, cuda), dev(B_st, cuda), Cg, m, n, k, alpha, beta, ta, tb)
    got = Cg.cpu().numpy().transpose(0, 2, 1).astype(np.float64)
    a64 = Ar.astype(np.float32).astype(np.float64)
    b64 = Br.astype(np.float32).astype(np.float64)
    c64 = Cr.astype(np.float32).astype(np.float64)
    if k == 0:   # the reference's quick return (magmablas/dgemm_batched_core.cu:211): C untouched
        assert np.array_equal(got, c64)
        return
    ref = alpha * a64 @ b64 + beta * c64
    for i in range(batch):
        assert err(got[i], ref[i], a64[i], b64[i], c64[i], k, alpha, beta) < 30 * eps, i


def test_gemm_fp32_tensor_core_beta_zero_ignores_c(cuda, fp32_tensor_core_tile):
    import magma_b200 as mb
    m = n = k = 40
    A = T.normal(4, 1, m * k).reshape(1, k, m).astype(np.float32)
    B = T.normal(4, 2, k * n).reshape(1, n, k).astype(np.float32)
    Cn = np.full((1, n, m), np.nan, np.float32)
    Cg = dev(Cn, cuda)
    mb.gemm_batched(dev(A, cuda), dev(B, cuda), Cg, m, n, k, 1.0, 0.0)
    got = Cg.cpu().numpy()
    assert np.isfinite(got).all()
    ref = (A[0].T.astype(np.float64) @ B[0].T.astype(np.float64))
    assert err(got[0].T, ref, A[0], B[0], np.zeros_like(ref), k, 1.0, 0.0) < 30 * np.finfo(np.float32).eps


def test_gemm_vbatched_fp32_tensor_core(cuda, fp32_tensor_core_tile):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    M, N, K = T.gemm_sizes(500, 1, 160, seed=13)
    rng = np.random.default_rng(8)
    As = [rng.standard_normal((int(k), int(m))).astype(np.float32) for m, k in zip(M, K)]
    Bs = [rng.standard_normal((int(n), int(k))).astype(np.float32) for k, n in zip(K, N)]
    Cs = [rng.standard_normal((int(n), int(m))).astype(np.float32) for m, n in zip(M, N)]
    gA, gB, gC = (VarBatch(x, cuda, torch.float32) for x in (As, Bs, Cs))
    mb.gemm_vbatched(gA, gB, gC, M, N, K, M, K, M, alpha=1.0, beta=0.5)
    eps = np.finfo(np.float32).eps
    for a, b, c, g, k in zip(As, Bs, Cs, gC.unpack(), K):
        a64, b64, c64 = a.T.astype(np.float64), b.T.astype(np.float64), c.T.astype(np.float64)
        ref = a64 @ b64 + 0.5 * c64
        assert err(g.T.astype(np.float64), ref, a64, b64, c64, int(k), 1.0, 0.5) < 30 * eps


@pytest.mark.parametrize("lower", [True, False])
def test_syrk_vbatched_fp32_tensor_core(cuda, fp32_tensor_core_tile, lower):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(29 + lower)
    count = 120
    Ns = rng.integers(1, 200, count).astype(np.int32)
    Ks = rng.integers(0, 90, count).astype(np.int32)
    lda = (Ns + 1).astype(np.int32)
    ldc = (Ns + 3).astype(np.int32)
    As = [rng.standard_normal((max(int(Ks[i]), 1), int(lda[i]))).astype(np.float32) for i in range(count)]
    Cs = [rng.standard_normal((int(Ns[i]), int(ldc[i]))).astype(np.float32) for i in range(count)]
    gA, gC = VarBatch(As, cuda, torch.float32), VarBatch(Cs, cuda, torch.float32)
    alpha, beta = 0.7, -0.4
    mb.syrk_vbatched(gA, gC, Ns, Ks, lda, ldc, alpha, beta, lower, False)
    out = gC.unpack()
    eps = np.finfo(np.float32).eps
    for i in range(count):
        n, k = int(Ns[i]), int(Ks[i])
        op = As[i][:k, :n].T.astype(np.float64)   # n x k
        c0 = Cs[i][:, :n].T.astype(np.float64)
        ref = alpha * op @ op.T + beta * c0
        got = out[i][:, :n].T.astype(np.float64)
        mask = np.tril(np.ones((n, n), bool)) if lower else np.triu(np.ones((n, n), bool))
        assert np.array_equal(got[~mask], c0[~mask].astype(np.float32).astype(np.float64)), i   # other triangle untouched
        den = np.sqrt(k + 2) * abs(alpha) * np.linalg.norm(op) ** 2 + 2 * abs(beta) * np.linalg.norm(c0)
        assert np.linalg.norm(np.where(mask, got - ref, 0)) / max(den, 1e-300) < 30 * eps, i
