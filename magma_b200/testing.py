"""Seeded input generators and error metrics for the batched solvers.

Inputs come from a project-owned counter-based PRNG (splitmix64 of
seed + (i+1)*golden), so any element of any stream can be regenerated on any
machine. Generators produce the synthetic workloads used by the tests and the
benchmark, with the shapes and value distributions of the reference's
testers (testing/magma_zgenerate.cpp, testing/testing_z*_batched.cpp):

* ``lu_uniform``      A, B ~ U[-1, 1]                 (plain FP64 LU + solve)
* ``gemm_vbatched``   M, N, K ~ U{lo..hi}, entries N(0,1), ld = roundup(M, 8)
* ``svd_logrand``     A = U diag(sigma) V^T, Haar U, V, sigma_i = exp(u_i ln(1/kappa))
                      (magma_generate_svd + Dist::logrand, magma_zgenerate.cpp:150-156, 197-266)
* ``spd_gram``        A = G G^T + n I, G ~ N(0,1)    (Cholesky workloads)

Layout: column-major batches of shape (batch, n, ld) (see magma_b200.api).
"""
from __future__ import annotations

import math

import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def stream_seed(seed: int, stream: int) -> np.uint64:
    """Independent sub-stream seed (stream 0 = A, 1 = B, 2.. = auxiliary)."""
    with np.errstate(over="ignore"):
        return _mix(np.array([np.uint64(seed) ^ (np.uint64(stream + 1) * _G)], dtype=np.uint64))[0]


def uniform01(seed: int, stream: int, count: int) -> np.ndarray:
    """count doubles in [0, 1) with 53 random bits each."""
    s = stream_seed(seed, stream)
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = _mix(s + idx * _G)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform11(seed: int, stream: int, count: int) -> np.ndarray:
    return 2.0 * uniform01(seed, stream, count) - 1.0


def normal(seed: int, stream: int, count: int) -> np.ndarray:
    """Box-Muller over two sub-streams."""
    u1 = uniform01(seed, 2 * stream + 100, count)
    u2 = uniform01(seed, 2 * stream + 101, count)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


def roundup(x, m):
    return ((np.asarray(x) + m - 1) // m) * m


# ---------------------------------------------------------------------------
def lu_uniform(batch: int, n: int, nrhs: int = 1, seed: int = 1, lda: int | None = None,
               ldb: int | None = None, m: int | None = None):
    """A (batch, n, lda) and B (batch, nrhs, ldb), entries U[-1,1]; padding is zero."""
    m = n if m is None else m
    lda = lda or max(1, m)
    ldb = ldb or max(1, m)
    A = np.zeros((batch, n, lda))
    A[:, :, :m] = uniform11(seed, 0, batch * n * m).reshape(batch, n, m)
    B = np.zeros((batch, nrhs, ldb))
    B[:, :, :m] = uniform11(seed, 1, batch * nrhs * m).reshape(batch, nrhs, m)
    return A, B


def gemm_sizes(count: int, lo: int = 8, hi: int = 128, seed: int = 2):
    u = uniform01(seed, 5, 3 * count).reshape(3, count)
    M, N, K = (lo + np.floor(u * (hi - lo + 1)).astype(np.int64)).clip(lo, hi)
    return M.astype(np.int32), N.astype(np.int32), K.astype(np.int32)


def haar(batch: int, n: int, seed: int, stream: int) -> np.ndarray:
    """Haar-distributed orthogonal matrices: QR of a Gaussian with R's diagonal made positive."""
    G = normal(seed, stream, batch * n * n).reshape(batch, n, n)
    Q, R = np.linalg.qr(G)
    d = np.sign(np.diagonal(R, axis1=1, axis2=2))
    d[d == 0] = 1.0
    return Q * d[:, None, :]


def svd_logrand(batch: int, n: int, kappa_lo: float = 1e2, kappa_hi: float = 1e6, nrhs: int = 4,
                seed: int = 3):
    """A = U diag(sigma) V^T with per-instance kappa_j log-uniform in [kappa_lo, kappa_hi].

    Returns (A (batch, n, n) column-major, B (batch, nrhs, n) ~ N(0,1), kappa (batch,))."""
    kap = np.exp(np.log(kappa_lo) + uniform01(seed, 6, batch) * (np.log(kappa_hi) - np.log(kappa_lo)))
    u = uniform01(seed, 7, batch * n).reshape(batch, n)
    sigma = np.exp(u * np.log(1.0 / kap)[:, None])
    U = haar(batch, n, seed, 8)
    V = haar(batch, n, seed, 9)
    A_rowmajor = (U * sigma[:, None, :]) @ np.transpose(V, (0, 2, 1))
    A = np.ascontiguousarray(np.transpose(A_rowmajor, (0, 2, 1)))   # column-major storage
    B = normal(seed, 10, batch * nrhs * n).reshape(batch, nrhs, n)
    return A, B, kap


def spd_gram(n: int, seed: int, index: int) -> np.ndarray:
    """A = G G^T + n I (column-major == row-major, symmetric)."""
    G = normal(seed, 1000 + index, n * n).reshape(n, n)
    return G @ G.T + n * np.eye(n)


# ---------------------------------------------------------------------------
def backward_error(A_cm: np.ndarray, X_cm: np.ndarray, B_cm: np.ndarray, n: int) -> np.ndarray:
    """Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), per instance and RHS.

    A_cm (batch, n, lda), X_cm and B_cm (batch, nrhs, ld) column-major."""
    A = np.transpose(A_cm[:, :n, :n], (0, 2, 1))       # row-major (batch, n, n)
    X = np.transpose(X_cm[:, :, :n], (0, 2, 1))        # (batch, n, nrhs)
    B = np.transpose(B_cm[:, :, :n], (0, 2, 1))
    R = B - A @ X
    anorm = np.abs(A).sum(axis=2).max(axis=1)          # inf-norm
    rn = np.abs(R).max(axis=1)
    xn = np.abs(X).max(axis=1)
    bn = np.abs(B).max(axis=1)
    return rn / (anorm[:, None] * xn + bn)


def lu_residual(A0_cm: np.ndarray, LU_cm: np.ndarray, ipiv: np.ndarray, m: int, n: int) -> np.ndarray:
    """MAGMA's getrf check ||P A - L U||_F / (||A||_F n) per instance (testing_zgetrf_batched.cpp:30-69)."""
    out = np.zeros(A0_cm.shape[0])
    k = min(m, n)
    for b in range(A0_cm.shape[0]):
        A = A0_cm[b, :n, :m].T.copy()
        LU = LU_cm[b, :n, :m].T
        L = np.tril(LU[:, :k], -1) + np.eye(m, k)
        U = np.triu(LU[:k, :])
        for j in range(k):
            p = ipiv[b, j] - 1
            if p != j:
                A[[j, p], :] = A[[p, j], :]
        out[b] = np.linalg.norm(A - L @ U) / (np.linalg.norm(A) * n)
    return out


def svd_logrand_torch(batch: int, n: int, kappa_lo: float = 1e2, kappa_hi: float = 1e6, nrhs: int = 4,
                      seed: int = 3, device="cuda"):
    """GPU version of svd_logrand for benchmark-sized batches (torch's seeded generator;
    U, V from the QR of Gaussians with R's diagonal made positive). Returns
    (A (batch, n, n) column-major, B (batch, nrhs, n), kappa (batch,)) as CUDA tensors."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)

    def haar_t():
        G = torch.randn(batch, n, n, dtype=torch.float64, device=device, generator=g)
        Q, R = torch.linalg.qr(G)
        d = torch.sign(torch.diagonal(R, dim1=1, dim2=2))
        d[d == 0] = 1.0
        return Q * d[:, None, :]

    kap = torch.exp(math.log(kappa_lo) + torch.rand(batch, dtype=torch.float64, device=device, generator=g)
                    * (math.log(kappa_hi) - math.log(kappa_lo)))
    sig = torch.exp(torch.rand(batch, n, dtype=torch.float64, device=device, generator=g)
                    * torch.log(1.0 / kap)[:, None])
    A_row = (haar_t() * sig[:, None, :]) @ haar_t().transpose(1, 2)
    A = A_row.transpose(1, 2).contiguous()
    B = torch.randn(batch, nrhs, n, dtype=torch.float64, device=device, generator=g)
    return A, B, kap


def backward_error_torch(A_cm, X_cm, B_cm):
    """Normwise backward error per instance and RHS on the GPU (FP64; used to verify results)."""
    A = A_cm.transpose(1, 2)
    X = X_cm.transpose(1, 2)
    Bm = B_cm.transpose(1, 2)
    R = Bm - A @ X
    anorm = A.abs().sum(dim=2).amax(dim=1)
    return R.abs().amax(dim=1) / (anorm[:, None] * X.abs().amax(dim=1) + Bm.abs().amax(dim=1))


def backward_error_vbatched_torch(A_flat, X_flat, B_flat, ns, nrhss, offA, offB):
    """Per-instance normwise backward error (max over RHS) of a variable-size batch on the GPU.

    A_flat, X_flat, B_flat are flat FP64 CUDA tensors; instance i is the n_i x n_i
    column-major block at offA[i] (lda = n_i) and its n_i x nrhs_i right-hand sides
    and solutions at offB[i] (ldb = n_i). Instances are grouped by order; RHS columns
    past an instance's own count are masked out. Returns a (batch,) FP64 tensor."""
    import torch

    ns, nrhss = np.asarray(ns), np.asarray(nrhss)
    dev = A_flat.device
    out = torch.zeros(len(ns), dtype=torch.float64, device=dev)
    for n in np.unique(ns):
        n = int(n)
        ids = np.nonzero(ns == n)[0]
        if n == 0:
            continue
        rmax = int(nrhss[ids].max())
        ia = torch.from_numpy(np.asarray(offA)[ids]).to(dev)[:, None] + torch.arange(n * n, device=dev)[None, :]
        A = A_flat[ia].reshape(len(ids), n, n).transpose(1, 2)                 # row-major view
        r = torch.arange(rmax, device=dev)
        live = r[None, :] < torch.from_numpy(nrhss[ids]).to(dev)[:, None]       # (k, rmax)
        ib = (torch.from_numpy(np.asarray(offB)[ids]).to(dev)[:, None, None] + (r * n)[None, :, None]
              + torch.arange(n, device=dev)[None, None, :])
        ib = torch.where(live[:, :, None], ib, torch.zeros_like(ib))
        X = torch.where(live[:, :, None], X_flat[ib], 0.0).transpose(1, 2)     # (k, n, rmax)
        B = torch.where(live[:, :, None], B_flat[ib], 0.0).transpose(1, 2)
        R = B - A @ X
        anorm = A.abs().sum(dim=2).amax(dim=1)
        be = R.abs().amax(dim=1) / (anorm[:, None] * X.abs().amax(dim=1) + B.abs().amax(dim=1))
        be = torch.where(live, be, torch.zeros_like(be))
        out[torch.from_numpy(ids).to(dev)] = be.amax(dim=1)
    return out


def lu_residual_torch(A0_cm, LU_cm, ipiv):
    """MAGMA's getrf check ||P A - L U||_F / (||A||_F n) per instance on the GPU, for square
    column-major (batch, n, n) tensors and 1-based LAPACK pivots (batch, n)."""
    import torch

    batch, n, _ = A0_cm.shape
    piv = np.asarray(ipiv.cpu() if hasattr(ipiv, "cpu") else ipiv).astype(np.int64) - 1
    perm = np.tile(np.arange(n), (batch, 1))
    rows = np.arange(batch)
    for j in range(n):                                   # LAPACK's sequential interchanges
        p = piv[:, j]
        pj, pp = perm[rows, j].copy(), perm[rows, p].copy()
        perm[rows, j], perm[rows, p] = pp, pj
    A = A0_cm.transpose(1, 2)                            # row-major views
    LU = LU_cm.transpose(1, 2)
    PA = torch.gather(A, 1, torch.from_numpy(perm).to(A.device)[:, :, None].expand(batch, n, n))
    eye = torch.eye(n, dtype=LU.dtype, device=LU.device)
    R = PA - (torch.tril(LU, -1) + eye) @ torch.triu(LU)
    return torch.linalg.norm(R, dim=(1, 2)) / (torch.linalg.norm(A, dim=(1, 2)) * n)
