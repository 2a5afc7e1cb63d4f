"""GPU tests of the mixed-precision batched solve (magma_dsgesv_batched).

Criterion: every instance's solution has normwise backward error
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-14 against the FP64
data; instances that refine keep A untouched; instances that fall back
(iter < 0) hold the FP64 LU, bit-identical to the oracle's dgetf2."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.fixture
def tensor_core_lu():
    """Every order n = 96..256 on the tensor-core LU (the built-in table keeps the
    CUDA-core LU at 96 and 128, where it measured faster), restored afterwards."""
    import ctypes as C

    from magma_b200 import _lib
    lib = _lib.load()
    count = lib.magma_b200_tuning_get(None, 0)
    vals = (C.c_int * count)()
    assert lib.magma_b200_tuning_get(vals, count) == count
    old = list(vals)
    vals[8] = 1                      # the tensor-core LU as a whole
    for i in range(13, 19):          # per order n = 96 + 32 (i - 13)
        vals[i] = 1
    assert lib.magma_b200_tuning_set(vals, count) == 0
    yield
    assert lib.magma_b200_tuning_set((C.c_int * count)(*old), count) == 0


@pytest.mark.parametrize("n,batch", [(16, 64), (48, 64), (64, 48), (100, 32), (256, 24), (400, 6)])
def test_dsgesv_svd_logrand(cuda, n, batch):
    import magma_b200 as mb
    A_np, B_np, kap = T.svd_logrand(batch, n, 1e2, 1e6, nrhs=4, seed=n)
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    X, ipiv, it, info = mb.dsgesv_batched(A, B)
    X, it, info = X.cpu().numpy(), it.cpu().numpy(), info.cpu().numpy()
    be = T.backward_error(A_np, X, B_np, n)
    assert be.max() <= 1e-14, (be.max(), it)
    assert np.array_equal(B.cpu().numpy(), B_np)             # B untouched
    ok = it >= 0
    assert ok.mean() > 0.5, it                               # most instances refine in FP32
    assert np.array_equal(A.cpu().numpy()[ok], A_np[ok])     # A untouched when refinement succeeded
    assert np.all(info == 0)
    if (~ok).any():                                          # fallback instances hold the FP64 LU
        O = A_np[~ok].copy()
        oip, oinf = oracle.dgetrf_batched(O, n)
        assert np.array_equal(A.cpu().numpy()[~ok], O)
        assert np.array_equal(ipiv.cpu().numpy()[~ok], oip)


def test_dsgesv_forced_fallbacks(cuda):
    import magma_b200 as mb
    n = 40
    A_np, B_np = T.lu_uniform(4, n, 2, seed=17)
    A_np[1, 3, 5] = 1e39                        # overflows single precision -> iter -2
    A_np[2, :, :] = 0.0                         # singular in both precisions -> iter -3, info > 0
    A_np[2, 0, 0] = 1.0
    A = dev(A_np, cuda)
    X, ipiv, it, info = mb.dsgesv_batched(A, dev(B_np, cuda))
    it, info = it.cpu().numpy(), info.cpu().numpy()
    assert it[0] >= 0 and it[3] >= 0
    assert it[1] == -2 and info[1] == 0
    assert it[2] == -3 and info[2] == 2
    O = A_np[[1, 2]].copy()
    oip, oinf = oracle.dgetrf_batched(O, n)
    assert np.array_equal(A.cpu().numpy()[[1, 2]], O)
    assert list(oinf) == [0, 2]
    be = T.backward_error(A_np[[0, 1, 3]], X.cpu().numpy()[[0, 1, 3]], B_np[[0, 1, 3]], n)
    assert be.max() <= 1e-14


@pytest.mark.parametrize("n,nrhs", [(37, 1), (130, 7), (255, 5)])
def test_dsgesv_rhs_counts(cuda, n, nrhs):
    """RHS counts that are not a multiple of the kernel's 4-column pass."""
    import magma_b200 as mb
    A_np, B_np, kap = T.svd_logrand(16, n, 1e2, 1e5, nrhs=nrhs, seed=7 * n + nrhs)
    X, ipiv, it, info = mb.dsgesv_batched(dev(A_np, cuda), dev(B_np, cuda))
    be = T.backward_error(A_np, X.cpu().numpy(), B_np, n)
    assert be.max() <= 1e-14, (be.max(), it)
    assert (it.cpu().numpy() >= 0).mean() > 0.5


@pytest.mark.parametrize("n", [96, 128, 160, 224, 256])
def test_dsgesv_tensor_core_lu(cuda, tensor_core_lu, n):
    """Orders 96..256 in steps of 32 factor on the tensor cores (TMEM-resident LU, split
    TF32): with kappa up to 1e6 the refinement must converge as from an FP32 LU, and
    where it does the single-precision pivots are LAPACK's on all but rare near-ties."""
    import magma_b200 as mb
    batch = 40
    A_np, B_np, kap = T.svd_logrand(batch, n, 1e2, 1e6, nrhs=4, seed=500 + n)
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    X, ipiv, it, info = mb.dsgesv_batched(A, B)
    X, it, ipiv = X.cpu().numpy(), it.cpu().numpy(), ipiv.cpu().numpy()
    be = T.backward_error(A_np, X, B_np, n)
    assert be.max() <= 1e-14, (be.max(), it)
    assert (it >= 0).mean() >= 0.9, it
    assert it[it >= 0].max() <= 8, it
    O = A_np.copy()
    oip, _ = oracle.dgetrf_batched(O, n)
    same = [np.array_equal(ipiv[i], oip[i]) for i in range(batch) if it[i] >= 0]
    # measured on B200: 92.5-97.5% of these instances (90.4% of a 512-instance C3 sample)
    assert np.mean(same) >= 0.9, np.mean(same)


def test_dsgesv_tensor_core_lu_fallbacks(cuda, tensor_core_lu):
    """The tensor-core path (n = 128) hands overflowing, NaN and singular instances to the
    FP64 fallback exactly as the CUDA-core path does."""
    import magma_b200 as mb
    n = 128
    A_np, B_np = T.lu_uniform(5, n, 3, seed=23)
    A_np[1, 3, 5] = 1e39                        # overflows single precision -> iter -2
    A_np[2, 7, 9] = np.nan                      # NaN -> iter -2, FP64 getrf carries the NaN
    A_np[3, 10, :] = 0.0                        # zero column 10 -> singular in both precisions
    A = dev(A_np, cuda)
    X, ipiv, it, info = mb.dsgesv_batched(A, dev(B_np, cuda))
    it, info = it.cpu().numpy(), info.cpu().numpy()
    assert it[0] >= 0 and it[4] >= 0
    assert it[1] == -2 and it[2] == -2 and it[3] == -3
    O = A_np[[1, 3]].copy()
    oip, oinf = oracle.dgetrf_batched(O, n)
    assert np.array_equal(A.cpu().numpy()[[1, 3]], O)
    assert list(info[[1, 3]]) == list(oinf) and oinf[1] == 11
    be = T.backward_error(A_np[[0, 1, 4]], X.cpu().numpy()[[0, 1, 4]], B_np[[0, 1, 4]], n)
    assert be.max() <= 1e-14


@pytest.mark.parametrize("n,nrhs,batch,chunks", [(96, 3, 37, 8), (40, 2, 9, 4), (256, 4, 20, 3)])
def test_dsgesv_host_pipelined_matches_device_call(cuda, n, nrhs, batch, chunks):
    """HostDsgesv (pinned host buffers, uploads/solves/read-backs overlapped chunk by chunk)
    gives the same X, iter and info, bit for bit, as one magma_dsgesv_batched call over the
    whole batch on device-resident data; one instance takes the FP64 fallback."""
    import torch
    import magma_b200 as mb
    from magma_b200.api import HostDsgesv, default_queue
    A_np, B_np, kap = T.svd_logrand(batch, n, 1e2, 1e6, nrhs=nrhs, seed=3 * n + batch)
    A_np[1, 2, 3] = 1e39                                      # overflows FP32 -> FP64 fallback
    X_d, ipiv_d, it_d, info_d = mb.dsgesv_batched(dev(A_np, cuda), dev(B_np, cuda))
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hA, hB = pin(A_np), pin(B_np)
    hX = torch.full((batch, nrhs, n), np.nan, dtype=torch.float64).pin_memory()
    hI = torch.full((batch,), 99, dtype=torch.int32).pin_memory()
    hF = torch.full((batch,), 99, dtype=torch.int32).pin_memory()
    solver = HostDsgesv(batch, n, nrhs, chunks=chunks)
    assert solver.bounds[0][0] == 0 and solver.bounds[-1][1] == batch and len(solver.bounds) <= chunks
    for _ in range(2):                                        # the staging buffers are reused
        hX.fill_(np.nan)
        solver(hA, hB, hX, hI, hF)
        default_queue().stream.synchronize()
        assert np.array_equal(hX.numpy(), X_d.cpu().numpy())
        assert np.array_equal(hI.numpy(), it_d.cpu().numpy())
        assert np.array_equal(hF.numpy(), info_d.cpu().numpy())
    assert hI.numpy()[1] == -2
    assert T.backward_error(A_np, hX.numpy(), B_np, n).max() <= 1e-14
    with pytest.raises(ValueError):
        solver(hA.clone(), hB, hX, hI, hF)                    # not pinned
