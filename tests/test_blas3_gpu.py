"""GPU tests of the batched BLAS-3 routines beside GEMM: magmablas_{d,s}trsm_vbatched*,
magmablas_{d,s}trmm_vbatched*, magmablas_{d,s}syrk_vbatched* and their fixed-size forms.

trsm / trmm (FP64) are BIT-IDENTICAL to the oracle, which restates the kernels' order of
operations (and is itself pinned to OpenBLAS dtrsm/dtrmm to rounding). FP32 and syrk use
the reference tester's criterion against a float64 product
(testing_zsyrk_vbatched.cpp, testing_ztrsm_vbatched.cpp: relative error below tol * eps)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps

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


# ------------------------------------------------------------------ fixed-size forms
@pytest.mark.parametrize("op", ["trsm", "trmm"])
@pytest.mark.parametrize("left,lower,trans,unit", COMBOS[::5] + [(True, True, False, False)])
def test_tri_batched_fixed_bit_identical(cuda, op, left, lower, trans, unit):
    """magmablas_dtrsm_batched / magmablas_dtrmm_batched (one size for all instances) give
    the oracle's bits, like the variable-size forms."""
    import torch

    from magma_b200.api import _vp, default_queue, ptr_array
    q = default_queue()
    rng = np.random.default_rng(31)
    m, n, batch = 70, 45, 30
    k = m if left else n
    lda, ldb = k + 2, m + 3
    A = rng.uniform(-1, 1, (batch, k, lda))
    idx = np.arange(k)
    A[:, idx, idx] += 2.0 * np.sign(A[:, idx, idx] + 1e-300) + 1.0
    B = rng.uniform(-1, 1, (batch, n, ldb))
    gA = torch.from_numpy(A).to(cuda)
    gB = torch.from_numpy(B).to(cuda)
    from magma_b200 import _lib
    f = getattr(q.lib, f"magmablas_d{op}_batched")
    pA, pB = ptr_array(gA), ptr_array(gB)          # kept alive until the call has run
    f(_lib.MagmaLeft if left else _lib.MagmaRight, _lib.MagmaLower if lower else _lib.MagmaUpper,
      _lib.MagmaTrans if trans else _lib.MagmaNoTrans, _lib.MagmaUnit if unit else _lib.MagmaNonUnit,
      m, n, 0.625, _vp(pA), lda, _vp(pB), ldb, batch, q.handle)
    out = gB.cpu().numpy()
    for b in range(batch):
        ref = B[b].copy()
        oracle.dtri(op == "trsm", left, lower, trans, unit, m, n, 0.625, A[b].copy(), ref)
        assert np.array_equal(out[b], ref), b


@pytest.mark.parametrize("lower,trans", [(True, False), (False, True)])
def test_syrk_batched_fixed(cuda, lower, trans):
    import torch

    from magma_b200 import _lib
    from magma_b200.api import _vp, default_queue, ptr_array
    q = default_queue()
    rng = np.random.default_rng(41)
    n, k, batch = 60, 37, 25
    rows, cols = (k, n) if trans else (n, k)
    lda, ldc = rows + 1, n + 2
    A = rng.standard_normal((batch, cols, lda))
    C0 = rng.standard_normal((batch, n, ldc))
    gA, gC = torch.from_numpy(A).to(cuda), torch.from_numpy(C0.copy()).to(cuda)
    pA, pC = ptr_array(gA), ptr_array(gC)          # kept alive until the call has run
    q.lib.magmablas_dsyrk_batched(_lib.MagmaLower if lower else _lib.MagmaUpper,
                                  _lib.MagmaTrans if trans else _lib.MagmaNoTrans, n, k, 0.7,
                                  _vp(pA), lda, -0.4, _vp(pC), ldc, batch, q.handle)
    out = gC.cpu().numpy()
    mask = np.tril(np.ones((n, n), bool)) if lower else np.triu(np.ones((n, n), bool))
    for b in range(batch):
        a = A[b][:cols, :rows].T
        op = a if not trans else a.T
        c0 = C0[b][:, :n].T
        ref = 0.7 * op @ op.T - 0.4 * c0
        got = out[b][:, :n].T
        assert syrk_err(np.where(mask, got, 0), np.where(mask, ref, 0), op, c0, k, 0.7, -0.4) < 30 * EPS
        assert np.array_equal(got[~mask], c0[~mask])
        assert np.array_equal(out[b][:, n:], C0[b][:, n:])


def test_fixed_forms_argument_errors(cuda, capfd):
    import torch

    from magma_b200 import _lib
    from magma_b200.api import _vp, default_queue, ptr_array
    q = default_queue()
    A = torch.zeros((1, 4, 4), dtype=torch.float64, device=cuda)
    pA = ptr_array(A)
    L, N, NU = _lib.MagmaLeft, _lib.MagmaNoTrans, _lib.MagmaNonUnit
    q.lib.magmablas_dtrsm_batched(L, _lib.MagmaLower, N, NU, 4, 4, 1.0, _vp(pA), 3, _vp(pA), 4, 1, q.handle)
    assert "parameter 9" in capfd.readouterr().err
    q.lib.magmablas_dtrmm_batched(L, _lib.MagmaLower, N, NU, 4, 4, 1.0, _vp(pA), 4, _vp(pA), 3, 1, q.handle)
    assert "parameter 11" in capfd.readouterr().err
    q.lib.magmablas_dsyrk_batched(_lib.MagmaLower, _lib.MagmaConjTrans, 4, 4, 1.0, _vp(pA), 4, 0.0, _vp(pA), 4, 1,
                                  q.handle)
    assert "parameter 2" in capfd.readouterr().err
    q.lib.magma_dsyrk_batched(_lib.MagmaLower, N, 4, 4, 1.0, _vp(pA), 3, 0.0, _vp(pA), 4, 1, q.handle)
    assert "parameter 7" in capfd.readouterr().err
