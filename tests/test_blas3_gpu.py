"""GPU tests of the variable-size batched BLAS-3 routines beside GEMM:
magmablas_{d,s}trsm_vbatched*, magmablas_{d,s}trmm_vbatched* and magmablas_{d,s}syrk_vbatched*.

trsm / trmm (FP64) are BIT-IDENTICAL to the oracle, which restates the kernels' order of
operations (and is itself pinned to OpenBLAS dtrsm/dtrmm to rounding). FP32 and syrk use
the reference tester's criterion against a float64 product
(testing_zsyrk_vbatched.cpp, testing_ztrsm_vbatched.cpp: relative error below tol * eps)."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu

COMBOS = [(left, lower, trans, unit) for left in (True, False) for lower in (True, False)
          for trans in (False, True) for unit in (False, True)]


def make_tri_batch(rng, count, lo, hi, left, dt=np.float64):
    M = rng.integers(lo, hi + 1, count).astype(np.int32)
    N = rng.integers(lo, hi + 1, count).astype(np.int32)
    M[:3], N[:3] = [1, hi, 33], [hi, 1, 64]
    K = M if left else N
    lda = (K + 3).astype(np.int32)
    ldb = (M + 2).astype(np.int32)
    As, Bs = [], []
    for i in range(count):
        a = rng.uniform(-1, 1, (K[i], lda[i]))
        a[np.arange(K[i]), np.arange(K[i])] += 2.0 * np.sign(a[np.arange(K[i]), np.arange(K[i])] + 1e-300) + 1.0
        a[:, K[i]:] = 7.0                                       # padding (never read)
        b = rng.uniform(-1, 1, (N[i], ldb[i]))
        As.append(a.astype(dt))
        Bs.append(b.astype(dt))
    return M, N, lda, ldb, As, Bs


@pytest.mark.parametrize("op", ["trsm", "trmm"])
@pytest.mark.parametrize("left,lower,trans,unit", COMBOS)
def test_tri_vbatched_bit_identical(cuda, op, left, lower, trans, unit):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(abs(hash((op, left, lower, trans, unit))) % 2**32)
    M, N, lda, ldb, As, Bs = make_tri_batch(rng, 40, 1, 100, left)
    gA, gB = VarBatch(As, cuda, torch.float64), VarBatch(Bs, cuda, torch.float64)
    alpha = 0.8125
    mb.tri_vbatched(op, gA, gB, M, N, lda, ldb, alpha, left, lower, trans, unit)
    out = gB.unpack()
    for i in range(len(Bs)):
        ref = Bs[i].copy()
        oracle.dtri(op == "trsm", left, lower, trans, unit, int(M[i]), int(N[i]), alpha, As[i].copy(), ref)
        assert np.array_equal(out[i], ref), (i, int(M[i]), int(N[i]), np.abs(out[i] - ref).max())


@pytest.mark.parametrize("op", ["trsm", "trmm"])
def test_tri_vbatched_large_and_forms(cuda, op):
    """Several 32-row tiles and column panels (m, n up to 300); the checked, _max_nocheck
    and _nocheck forms give the same bits."""
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(5)
    for left, lower, trans in ((True, True, False), (False, False, True), (True, False, True)):
        M, N, lda, ldb, As, Bs = make_tri_batch(rng, 12, 100, 300, left)
        outs = []
        for form in ("checked", "max", "nocheck"):
            gA, gB = VarBatch(As, cuda, torch.float64), VarBatch(Bs, cuda, torch.float64)
            mx = (int(M.max()), int(N.max())) if form == "max" else None
            mb.tri_vbatched(op, gA, gB, M, N, lda, ldb, -1.5, left, lower, trans, False, max_sizes=mx,
                            checked=(form == "checked"))
            outs.append(gB.unpack())
        for i in range(len(Bs)):
            ref = Bs[i].copy()
            oracle.dtri(op == "trsm", left, lower, trans, False, int(M[i]), int(N[i]), -1.5, As[i].copy(), ref)
            for o in outs:
                assert np.array_equal(o[i], ref), (left, lower, trans, i)


@pytest.mark.parametrize("op", ["trsm", "trmm"])
def test_tri_vbatched_fp32(cuda, op):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(9)
    for left, lower, trans, unit in COMBOS[::3]:
        M, N, lda, ldb, As, Bs = make_tri_batch(rng, 20, 1, 90, left, np.float32)
        gA, gB = VarBatch(As, cuda, torch.float32), VarBatch(Bs, cuda, torch.float32)
        mb.tri_vbatched(op, gA, gB, M, N, lda, ldb, 0.5, left, lower, trans, unit)
        out = gB.unpack()
        for i in range(len(Bs)):
            ref = Bs[i].astype(np.float64)
            oracle.dtri(op == "trsm", left, lower, trans, unit, int(M[i]), int(N[i]), 0.5, As[i].astype(np.float64),
                        ref)
            scale = max(1.0, np.abs(ref).max())
            assert np.abs(out[i] - ref).max() < 1e-4 * scale, (left, lower, trans, unit, i)


def test_tri_vbatched_alpha_zero_and_empty(cuda):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(3)
    M, N, lda, ldb, As, Bs = make_tri_batch(rng, 6, 1, 40, True)
    M[2] = 0                                                     # an empty instance is skipped
    for op in ("trsm", "trmm"):
        gA, gB = VarBatch(As, cuda, torch.float64), VarBatch(Bs, cuda, torch.float64)
        mb.tri_vbatched(op, gA, gB, M, N, lda, ldb, 0.0, True, True, False, False)
        out = gB.unpack()
        for i in range(len(Bs)):
            assert np.all(out[i][:, :M[i]] == 0.0)
            assert np.array_equal(out[i][:, M[i]:], Bs[i][:, M[i]:])


def test_tri_vbatched_argument_errors(cuda, capfd):
    import torch

    from magma_b200 import _lib
    from magma_b200.api import VarBatch, _vp, default_queue
    q = default_queue()
    A = VarBatch([np.eye(4)], cuda, torch.float64)
    B = VarBatch([np.ones((4, 4))], cuda, torch.float64)
    f = q.lib.magmablas_dtrsm_vbatched

    def call(side=_lib.MagmaLeft, uplo=_lib.MagmaLower, tr=_lib.MagmaNoTrans, dg=_lib.MagmaNonUnit, m=4, n=4,
             lda=4, ldb=4):
        dm, dn, dla, dlb = B.ints([m]), B.ints([n]), B.ints([lda]), B.ints([ldb])
        f(side, uplo, tr, dg, _vp(dm), _vp(dn), 1.0, _vp(A.ptrs), _vp(dla), _vp(B.ptrs), _vp(dlb), 1, q.handle)
        return capfd.readouterr().err

    assert "parameter 1" in call(side=7)
    assert "parameter 2" in call(uplo=7)
    assert "parameter 3" in call(tr=7)
    assert "parameter 4" in call(dg=7)
    assert "parameter 5" in call(m=-1)
    assert "parameter 6" in call(n=-1)
    assert "parameter 9" in call(lda=3)
    assert "parameter 11" in call(ldb=3)
    assert call() == ""


# ------------------------------------------------------------------------ syrk
def syrk_err(got, ref, a, c0, k, alpha, beta):
    den = np.sqrt(k + 2) * abs(alpha) * np.linalg.norm(a) ** 2 + 2 * abs(beta) * np.linalg.norm(c0)
    return np.linalg.norm(got - ref) / max(den, 1e-300)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("lower,trans", [(True, False), (True, True), (False, False), (False, True)])
def test_syrk_vbatched(cuda, dt, lower, trans):
    import torch

    import magma_b200 as mb
    from magma_b200.api import VarBatch
    rng = np.random.default_rng(17 + 2 * lower + trans)
    count = 300
    Ns = rng.integers(1, 130, count).astype(np.int32)
    Ks = rng.integers(0, 130, count).astype(np.int32)
    Ns[:2], Ks[:2] = [128, 1], [0, 129]
    rows = Ks if trans else Ns
    cols = Ns if trans else Ks
    lda = (rows + 1).astype(np.int32)
    ldc = (Ns + 3).astype(np.int32)
    As = [rng.standard_normal((max(cols[i], 1), lda[i])).astype(dt) for i in range(count)]
    Cs = [rng.standard_normal((Ns[i], ldc[i])).astype(dt) for i in range(count)]
    tdt = torch.float64 if dt == np.float64 else torch.float32
    gA, gC = VarBatch(As, cuda, tdt), VarBatch(Cs, cuda, tdt)
    alpha, beta = 0.7, -0.4
    mb.syrk_vbatched(gA, gC, Ns, Ks, lda, ldc, alpha, beta, lower, trans)
    out = gC.unpack()
    eps = np.finfo(dt).eps
    for i in range(count):
        n, k = int(Ns[i]), int(Ks[i])
        a = As[i][:cols[i], :rows[i]].T.astype(np.float64)       # rows x cols
        op = a if not trans else a.T                                # n x k
        c0 = Cs[i][:, :n].T.astype(np.float64)
        ref = alpha * op @ op.T + beta * c0
        got = out[i][:, :n].T.astype(np.float64)
        mask = np.tril(np.ones((n, n), bool)) if lower else np.triu(np.ones((n, n), bool))
        assert syrk_err(np.where(mask, got, 0), np.where(mask, ref, 0), op, c0, k, alpha, beta) < 30 * eps, i
        assert np.array_equal(got[~mask], c0[~mask].astype(dt).astype(np.float64)), i   # other triangle untouched
        assert np.array_equal(out[i][:, n:], Cs[i][:, n:])                               # padding untouched


def test_syrk_vbatched_argument_errors(cuda, capfd):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    A = VarBatch([np.eye(4)], cuda)
    C = VarBatch([np.eye(4)], cuda)
    mb.syrk_vbatched(A, C, [-1], [4], [4], [4])
    assert "parameter 3" in capfd.readouterr().err
    mb.syrk_vbatched(A, C, [4], [-1], [4], [4])
    assert "parameter 4" in capfd.readouterr().err
    mb.syrk_vbatched(A, C, [4], [4], [3], [4])
    assert "parameter 7" in capfd.readouterr().err
    mb.syrk_vbatched(A, C, [4], [4], [4], [3])
    assert "parameter 10" in capfd.readouterr().err
