"""GPU tests of the batched Householder QR (magma_dgeqrf_batched).

Checks follow the reference's testing_zgeqrf_batched.cpp: ||R - Q^T A||_1 / (N ||A||_1)
and ||I - Q^T Q||_1 / N below 30 eps; in addition the reflectors, R and tau agree with
the oracle's dgeqr2 restatement BIT FOR BIT: the oracle writes out the kernel's
summation order (rows dealt to P lanes, ascending fma chains, pairwise tree), and is
itself pinned to LAPACK dgeqrf to rounding."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def form_q(h, tau, m, k):
    """Q = H(1) ... H(k) from LAPACK's representation (h column-major (n, lda))."""
    Q = np.eye(m)
    for i in reversed(range(k)):
        v = np.zeros(m)
        v[i] = 1.0
        v[i + 1:m] = h[i, i + 1:m]
        Q -= tau[i] * np.outer(v, v @ Q)
    return Q


def qr_errors(A0, h, tau, m, n):
    k = min(m, n)
    A = A0[:, :m].T                                   # m x n, row-major
    Q = form_q(h, tau, m, k)[:, :k]                   # the m x min(m,n) factor, as the reference forms it
    R = np.triu(h[:, :m].T)[:k, :]
    e1 = np.abs(R - Q.T @ A).sum(axis=0).max() / (n * np.abs(A).sum(axis=0).max())
    e2 = np.abs(np.eye(k) - Q.T @ Q).sum(axis=0).max() / n
    return e1, e2


@pytest.mark.parametrize("m,n,batch,lda", [(1, 1, 7, 1), (8, 8, 50, 8), (32, 16, 40, 32), (40, 17, 30, 45),
                                           (64, 64, 20, 64), (100, 32, 16, 100), (128, 64, 10, 130),
                                           (200, 50, 8, 200), (256, 64, 6, 256), (256, 1, 6, 256),
                                           (10, 30, 12, 10), (20, 64, 8, 24), (5, 3, 9, 5), (17, 17, 9, 17),
                                           (33, 40, 9, 35), (49, 20, 9, 49), (64, 8, 9, 64), (16, 33, 9, 16),
                                           # more than 64 columns: panels of 64, earlier reflectors replayed
                                           (64, 100, 6, 64), (128, 130, 4, 128), (256, 200, 3, 256),
                                           (100, 256, 3, 101), (30, 200, 4, 30), (256, 300, 2, 260),
                                           (200, 129, 4, 200),
                                           # 257..512 rows: 64 rows a lane, panels of 32 columns
                                           (300, 40, 3, 300), (512, 70, 2, 512), (400, 400, 2, 401), (257, 3, 4, 257),
                                           # 513..1024 rows: 16 lanes a column, 64 rows a lane, panels of 16 columns
                                           (513, 5, 3, 513), (700, 40, 2, 703), (1024, 33, 2, 1024),
                                           (600, 600, 1, 600), (1000, 1100, 1, 1001)])
def test_geqrf_matches_oracle(cuda, m, n, batch, lda):
    import magma_b200 as mb
    rng = np.random.default_rng(1000 * m + n)
    A_np = rng.uniform(-1, 1, (batch, n, lda))
    A = dev(A_np, cuda)
    tau = mb.dgeqrf_batched(A, m).cpu().numpy()
    G = A.cpu().numpy()
    O = A_np.copy()
    tau_o = oracle.dgeqrf_batched(O, m)
    k = min(m, n)
    assert np.array_equal(G[:, :, m:], A_np[:, :, m:])            # padding rows untouched
    assert np.array_equal(G, O)                                    # the oracle restates the kernel's order
    assert np.array_equal(tau[:, :k], tau_o[:, :k])
    assert np.abs(G - O).max() < 64 * max(m, n) * EPS
    assert np.abs(tau[:, :k] - tau_o[:, :k]).max() < 64 * max(m, n) * EPS
    for b in range(batch):
        e1, e2 = qr_errors(A_np[b], G[b], tau[b], m, n)
        assert e1 < 30 * EPS and e2 < 30 * EPS, (b, e1, e2)


def test_geqrf_zero_and_ill_conditioned_columns(cuda):
    """A zero column below the diagonal gives tau = 0 (H = I); a rank-deficient instance
    still gives an orthogonal Q; other instances are unaffected."""
    import magma_b200 as mb
    m, n, batch = 48, 24, 5
    rng = np.random.default_rng(7)
    A_np = rng.uniform(-1, 1, (batch, n, m))
    A_np[1, 3, 4:] = 0.0                        # column 3 zero below row 3 -> x = 0 at step 3
    A_np[1, 3, :4] = 0.0
    A_np[2, 10] = A_np[2, 9]                    # two equal columns: rank deficient
    A_np[3] *= 1e-150                           # tiny but representable entries
    A = dev(A_np, cuda)
    tau = mb.dgeqrf_batched(A, m).cpu().numpy()
    G = A.cpu().numpy()
    O = A_np.copy()
    tau_o = oracle.dgeqrf_batched(O, m)
    assert np.all(np.isfinite(G)) and np.all(np.isfinite(tau))
    assert np.array_equal(G, O) and np.array_equal(tau, tau_o)     # bit-identical, even the noise column
    well = [0, 1, 3, 4]      # instance 2's column 10 is rounding noise after step 9: its reflector is arbitrary
    assert np.abs(tau[well] - tau_o[well]).max() < 64 * m * EPS
    assert tau[1, 3] == 0.0 and tau_o[1, 3] == 0.0
    for b in range(batch):
        e1, e2 = qr_errors(A_np[b], G[b], tau[b], m, n)
        assert e2 < 30 * EPS, (b, e2)
        assert e1 < 30 * EPS, (b, e1)


def test_geqrf_argument_errors(cuda):
    import torch
    from magma_b200 import _lib
    from magma_b200.api import default_queue, ptr_array
    q = default_queue()
    A = torch.zeros((2, 4, 8), dtype=torch.float64, device=cuda)
    tau = torch.zeros((2, 4), dtype=torch.float64, device=cuda)
    info = torch.full((2,), 5, dtype=torch.int32, device=cuda)
    pA, pT = ptr_array(A), ptr_array(tau)
    f = q.lib.magma_dgeqrf_batched
    vp = lambda t: t.data_ptr()
    assert f(-1, 4, vp(pA), 8, vp(pT), vp(info), 2, q.handle) == -1
    assert f(8, -1, vp(pA), 8, vp(pT), vp(info), 2, q.handle) == -2
    assert f(8, 4, vp(pA), 7, vp(pT), vp(info), 2, q.handle) == -4
    torch.cuda.synchronize()
    assert info.cpu().tolist() == [0, 0]                            # zeroed before the checks
    assert f(8, 0, vp(pA), 8, vp(pT), vp(info), 2, q.handle) == 0  # quick return
    # more than 1024 rows is refused before any work (the arrays here are far too small for
    # such a matrix, and nothing reads them)
    assert f(1025, 4, vp(pA), 1025, vp(pT), vp(info), 2, q.handle) == _lib.MAGMA_ERR_NOT_SUPPORTED
