"""GPU tests at the benchmark's full instance counts.

C3: 2,048 x (256x256), A = U diag(sigma) V^T with kappa log-uniform in [1e2, 1e6], 4 RHS.
  * plain FP64 (magma_dgesv_batched): pivots and info identical to the reference's CPU
    LAPACK loop on every instance, MAGMA's getrf criterion ||PA - LU||_F / (||A||_F n)
    < 30 eps (testing/testing_zgetrf_batched.cpp:253), backward error <= 1e-14;
  * mixed (magma_dsgesv_batched): backward error <= 1e-14 and info 0 on every instance
    (the criterion of testing/testing_zcgesv_gpu.cpp:111-118 tightened to the metric's
    bar), A untouched where refinement converged, and the FP64 fallback instances
    holding exactly the plain FP64 path's factors and pivots.
C4: 50,000 SPD instances, n power-law on [4, 512], 1-8 RHS (the benchmark's generator):
  FP64 posv bit-identical to the oracle on a sample that includes the 50 largest orders,
  backward error <= 1e-14 and info 0 on every instance, for the FP64 and the mixed arms.
"""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def test_c3_full_fp64_and_mixed(cuda):
    import torch

    import magma_b200 as mb

    batch, n, nrhs = 2048, 256, 4
    A0, B0, kap = T.svd_logrand_torch(batch, n, 1e2, 1e6, nrhs, seed=3, device=cuda)
    # plain FP64
    A, B = A0.clone(), B0.clone()
    ipiv, info = mb.dgesv_batched(A, B)
    torch.cuda.synchronize()
    L = A0.cpu().numpy().copy()
    lip, linf = oracle.lapack_dgetrf_batched(L, n)
    assert np.array_equal(ipiv.cpu().numpy(), lip), "pivots differ from the LAPACK loop"
    assert np.array_equal(info.cpu().numpy(), linf) and not linf.any()
    res = T.lu_residual_torch(A0, A, ipiv)
    assert res.max().item() < 30 * EPS, res.max().item()
    be = T.backward_error_torch(A0, B, B0)
    assert be.max().item() <= 1e-14, be.max().item()
    LU64, piv64 = A, ipiv.clone()
    # mixed precision
    Am = A0.clone()
    X, ipm, it, infm = mb.dsgesv_batched(Am, B0)
    torch.cuda.synchronize()
    be = T.backward_error_torch(A0, X, B0)
    assert be.max().item() <= 1e-14, be.max().item()
    assert not infm.any().item()
    ok = it >= 0
    assert ok.float().mean().item() >= 0.95, torch.unique(it, return_counts=True)
    assert torch.equal(Am[ok], A0[ok]), "A modified where refinement converged"
    if (~ok).any():
        assert torch.equal(Am[~ok], LU64[~ok]) and torch.equal(ipm[~ok], piv64[~ok])


def test_c4_full_fp64_and_mixed(cuda):
    import torch

    import bench
    from magma_b200.api import Queue

    stream = torch.cuda.Stream(cuda)
    with torch.cuda.stream(stream):
        W = bench.C4CholVbatched(cuda)
        q = Queue(stream, cuda.index or 0)
        W.restore(0)
        assert W._raw_fp64(q) == 0
        q.sync()
        g, ok = bench.accuracy_gate("fp64", W._bwd_all(W.B), W.info[:W.batch])
        assert ok, g
        # bit-identical to the oracle on a sample: the 50 largest orders and every 250th instance
        sample = sorted(set(np.argsort(W.n)[-50:].tolist() + list(range(0, W.batch, 250))))
        A0, B0 = W.A0.cpu().numpy(), W.B0.cpu().numpy()
        GA, GB = W.A.cpu().numpy(), W.B.cpu().numpy()
        ns, nr = W.n[sample], W.nrhs[sample]
        As = [A0[W.offA[i]:W.offA[i] + W.n[i] ** 2].reshape(W.n[i], W.n[i]).copy() for i in sample]
        Bs = [B0[W.offB[i]:W.offB[i] + W.n[i] * W.nrhs[i]].reshape(W.nrhs[i], W.n[i]).copy() for i in sample]
        oinf = oracle.dposv_vbatched(As, Bs, ns, nr, ns, ns)
        assert not np.any(oinf)
        for j, i in enumerate(sample):
            k = int(W.n[i])
            got = GA[W.offA[i]:W.offA[i] + k * k].reshape(k, k)
            assert np.array_equal(np.tril(got.T), np.tril(As[j].T)), i
            assert np.array_equal(GB[W.offB[i]:W.offB[i] + k * W.nrhs[i]], Bs[j].reshape(-1)), i
        # mixed arm: FP32 factor + FP64 refinement
        W.restore_alt(0)
        assert W._raw_mixed(q) == 0
        q.sync()
        g, ok = bench.accuracy_gate("mixed", W._bwd_all(W.X), W.info[:W.batch])
        assert ok, g
