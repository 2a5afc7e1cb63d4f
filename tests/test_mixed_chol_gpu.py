"""GPU tests of the variable-size mixed-precision Cholesky solve (magma_dsposv_vbatched).

Criterion (as magma_dsposv_gpu, src/zcposv_gpu.cpp:134-330): every solution has
normwise backward error <= 1e-14 against the FP64 data; refined instances leave
A untouched; instances that fall back to FP64 hold the FP64 Cholesky factor,
bit-identical to the oracle, and their info is LAPACK's."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def _mixed_batch(count, seed, n_hi=512):
    rng = np.random.default_rng(seed)
    ns = np.concatenate([[1, 31, 32, 33, 64, 65, 200, n_hi], rng.integers(2, n_hi + 1, count - 8)])
    nrhs = rng.integers(1, 9, count)
    As = [np.ascontiguousarray(T.spd_gram(int(n), seed, i)) for i, n in enumerate(ns)]
    Bs = [rng.standard_normal((int(r), int(n))) for n, r in zip(ns, nrhs)]
    return ns, nrhs, As, Bs


def _bwd(A, X, B):
    """max over RHS of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf); arrays (cols, n)."""
    R = B.T - A @ X.T
    an = np.abs(A).sum(axis=1).max()
    return float((np.abs(R).max(axis=0) / (an * np.abs(X.T).max(axis=0) + np.abs(B.T).max(axis=0))).max())


@pytest.mark.parametrize("checked", [True, False])
def test_dsposv_vbatched_backward_error(cuda, checked):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    ns, nrhs, As, Bs = _mixed_batch(60, 21)
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    ms = (int(ns.max()), int(nrhs.max())) if not checked else None
    X, it, info = mb.dsposv_vbatched(gA, gB, ns, nrhs, max_sizes=ms)
    it, info = it.cpu().numpy(), info.cpu().numpy()
    Xs = X.unpack()
    assert np.all(info == 0)
    assert np.all(it >= 0), it                      # SPD and well conditioned: all refine in FP32
    for i in range(len(ns)):
        assert _bwd(As[i], Xs[i], Bs[i]) <= 1e-14, (i, ns[i])
    Aout = gA.unpack()
    for i in range(len(ns)):
        assert np.array_equal(Aout[i], As[i])       # A untouched
    for i in range(len(Bs)):
        assert np.array_equal(gB.unpack()[i], Bs[i])


def test_dsposv_vbatched_fallbacks(cuda):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    ns = np.array([40, 70, 90, 20])
    nrhs = np.array([2, 1, 3, 4])
    As = [np.ascontiguousarray(T.spd_gram(int(n), 5, i)) for i, n in enumerate(ns)]
    As[1][3, 3] = 1e39                              # overflows single precision -> iter -2, FP64 succeeds
    As[2][10, 10] = -5.0                            # not positive definite -> iter -3, info 11 in FP64
    rng = np.random.default_rng(3)
    Bs = [rng.standard_normal((int(r), int(n))) for n, r in zip(ns, nrhs)]
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    X, it, info = mb.dsposv_vbatched(gA, gB, ns, nrhs)
    it, info = it.cpu().numpy(), info.cpu().numpy()
    assert it[0] >= 0 and it[3] >= 0
    assert it[1] == -2 and it[2] == -3
    O = [As[1].copy(), As[2].copy()]
    Ob = [np.zeros((1, 70)), np.zeros((1, 90))]
    oinfo = oracle.dposv_vbatched(O, Ob, [70, 90], [1, 1], [70, 90], [70, 90], solve=False, upper=False)
    assert list(info[[1, 2]]) == list(oinfo)
    assert oinfo[1] == 11
    Aout = gA.unpack()
    assert np.array_equal(np.tril(Aout[1]), np.tril(O[0]))   # FP64 factor, bit-identical to the oracle
    Xs = X.unpack()
    for i in (0, 1, 3):
        assert _bwd(As[i], Xs[i], Bs[i]) <= 1e-14, i


def test_dsposv_vbatched_argument_errors(cuda):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    gA = VarBatch([np.eye(4), np.eye(3)], cuda)
    gB = VarBatch([np.ones((1, 4)), np.ones((1, 3))], cuda)
    with pytest.raises(ValueError, match="-2"):
        mb.dsposv_vbatched(gA, gB, [4, -3], [1, 1])
    with pytest.raises(ValueError, match="-5"):
        mb.dsposv_vbatched(gA, gB, [4, 3], [1, 1], lda=[4, 2])
