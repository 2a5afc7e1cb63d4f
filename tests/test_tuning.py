"""The kernel-variant tuning table (magma_b200_tuning_* / magma_b200_autotune).

CPU part: get / set / save / load round trips and argument checks (host only).
GPU part: every GEMM tile variant gives bit-identical results, and the
autotuner runs and leaves a valid table."""
import ctypes as C

import numpy as np
import pytest

from magma_b200 import _lib

N_VALUES = 21


def _get(lib):
    v = (C.c_int * N_VALUES)()
    assert lib.magma_b200_tuning_get(v, N_VALUES) == N_VALUES
    return list(v)


def _set(lib, vals):
    arr = (C.c_int * len(vals))(*vals)
    return lib.magma_b200_tuning_set(arr, len(vals))


def test_tuning_roundtrip(tmp_path):
    lib = _lib.load()
    assert lib.magma_b200_tuning_get(None, 0) == N_VALUES           # size query
    orig = _get(lib)
    try:
        new = [0, 1, 2, 0, 2, 1, 0, 0, 0, 1, 0, 1, 1, 1, 0, 1, 1, 0, 1, 0, 0]
        assert _set(lib, new) == 0 and _get(lib) == new
        f = tmp_path / "tune.txt"
        assert lib.magma_b200_tuning_save(str(f).encode()) == 0
        assert f.read_text().split()[0] == "magma_b200_tuning_v5"
        assert _set(lib, orig) == 0 and _get(lib) == orig
        assert lib.magma_b200_tuning_load(str(f).encode()) == 0 and _get(lib) == new
        # rejected: wrong count, out-of-range values, unreadable or malformed files
        assert _set(lib, new[:-3]) == _lib.MAGMA_ERR_ILLEGAL_VALUE   # 18: no table has that size
        assert _set(lib, [4] + new[1:]) == _lib.MAGMA_ERR_ILLEGAL_VALUE      # FP64 tiles: 0..3
        assert _set(lib, new[:4] + [4] + new[5:]) == _lib.MAGMA_ERR_ILLEGAL_VALUE   # FP32 tiles: 0..3
        assert _set(lib, new[:4] + [3] + new[5:]) == 0 and _get(lib)[4] == 3
        assert _set(lib, [3] + new[1:]) == 0 and _get(lib)[0] == 3
        assert _set(lib, new) == 0
        assert _set(lib, new[:-1] + [2]) == _lib.MAGMA_ERR_ILLEGAL_VALUE
        # 9-, 13-, 19- and 20-value tables (saved before the later entries existed) set their part only
        assert _set(lib, orig[:9]) == 0 and _get(lib) == orig[:9] + new[9:]
        assert _set(lib, orig[:13]) == 0 and _get(lib) == orig[:13] + new[13:]
        assert _set(lib, orig[:19]) == 0 and _get(lib) == orig[:19] + new[19:]
        assert _set(lib, orig[:20]) == 0 and _get(lib) == orig[:20] + new[20:]
        v1 = tmp_path / "v1.txt"
        v1.write_text("magma_b200_tuning_v1\n" + " ".join(map(str, new[:9])) + "\n")
        assert lib.magma_b200_tuning_load(str(v1).encode()) == 0 and _get(lib) == new[:9] + orig[9:20] + new[20:]
        v2 = tmp_path / "v2.txt"
        v2.write_text("magma_b200_tuning_v2\n" + " ".join(map(str, new[:13])) + "\n")
        assert lib.magma_b200_tuning_load(str(v2).encode()) == 0 and _get(lib) == new[:13] + orig[13:20] + new[20:]
        assert _set(lib, new) == 0
        v3 = tmp_path / "v3.txt"
        v3.write_text("magma_b200_tuning_v3\n" + " ".join(map(str, orig[:19])) + "\n")
        assert lib.magma_b200_tuning_load(str(v3).encode()) == 0 and _get(lib) == orig[:19] + new[19:]
        assert _set(lib, new) == 0
        v4 = tmp_path / "v4.txt"
        v4.write_text("magma_b200_tuning_v4\n" + " ".join(map(str, orig[:20])) + "\n")
        assert lib.magma_b200_tuning_load(str(v4).encode()) == 0 and _get(lib) == orig[:20] + new[20:]
        assert _set(lib, new) == 0
        assert lib.magma_b200_tuning_load(str(tmp_path / "missing").encode()) == _lib.MAGMA_ERR_ILLEGAL_VALUE
        bad = tmp_path / "bad.txt"
        bad.write_text("magma_b200_tuning_v1\n0 1 2\n")
        assert lib.magma_b200_tuning_load(str(bad).encode()) == _lib.MAGMA_ERR_ILLEGAL_VALUE
        assert _get(lib) == new
    finally:
        _set(lib, orig)


@pytest.mark.gpu
def test_gemm_variants_bit_identical(cuda):
    import torch

    import magma_b200 as mb
    from magma_b200 import testing as T
    from magma_b200.api import VarBatch
    lib = _lib.load()
    orig = _get(lib)
    M, N, K = T.gemm_sizes(600, 1, 100, seed=9)
    rng = np.random.default_rng(4)
    outs = {}
    try:
        for prec, dt in (("d", torch.float64), ("s", torch.float32)):
            As = [rng.standard_normal((int(k), int(m))) for m, k in zip(M, K)]
            Bs = [rng.standard_normal((int(n), int(k))) for k, n in zip(K, N)]
            Cs = [rng.standard_normal((int(n), int(m))) for m, n in zip(M, N)]
            for v in range(4):
                vals = list(orig)
                for b in range(4):
                    vals[(0 if prec == "d" else 4) + b] = v
                assert _set(lib, vals) == 0
                gA, gB, gC = VarBatch(As, cuda, dt), VarBatch(Bs, cuda, dt), VarBatch(Cs, cuda, dt)
                mb.gemm_vbatched(gA, gB, gC, M, N, K, M, K, M, alpha=1.0, beta=0.5)
                torch.cuda.synchronize()
                outs[(prec, v)] = gC.buf.cpu().numpy()
            assert np.array_equal(outs[(prec, 0)], outs[(prec, 1)])
            assert np.array_equal(outs[(prec, 0)], outs[(prec, 2)])
            if prec == "d":   # the FP64 tensor-core tile
                assert np.array_equal(outs[(prec, 0)], outs[(prec, 3)])
            else:             # the FP32 tcgen05 tile: split TF32, within the tester's bound instead
                ref3 = [a.T @ b.T + 0.5 * c.T for a, b, c in zip(As, Bs, Cs)]
                g3 = VarBatch(Cs, cuda, dt)
                g3.buf = torch.from_numpy(outs[(prec, 3)])
                eps = np.finfo(np.float32).eps
                for r, gg, a, b, c, kk in zip(ref3, g3.unpack(), As, Bs, Cs, K):
                    num = np.linalg.norm(gg.T - r)
                    den = np.sqrt(kk + 2) * np.linalg.norm(a) * np.linalg.norm(b) + 2 * 0.5 * np.linalg.norm(c)
                    assert num / den < 30 * eps
            # and the result is right (FP64 reference)
            ref = [a.T @ b.T + 0.5 * c.T for a, b, c in zip(As, Bs, Cs)]
            got = VarBatch(Cs, cuda, dt)
            got.buf = torch.from_numpy(outs[(prec, 0)])
            tol = 1e-12 if prec == "d" else 1e-4
            for r, g in zip(ref, got.unpack()):
                assert np.abs(g.T - r).max() <= tol * max(1.0, np.abs(r).max()) * 128
    finally:
        _set(lib, orig)


@pytest.mark.gpu
def test_autotune_runs(cuda, tmp_path):
    from magma_b200.api import default_queue
    lib = _lib.load()
    orig = _get(lib)
    try:
        q = default_queue()
        assert lib.magma_b200_autotune(q.handle) == 0
        vals = _get(lib)
        assert all(0 <= v <= 3 for v in vals[:8])
        assert all(v in (0, 1) for v in vals[8:])
        f = tmp_path / "tuned.txt"
        assert lib.magma_b200_tuning_save(str(f).encode()) == 0
    finally:
        _set(lib, orig)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [100, 256, 300, 700])
def test_lu_update_variants_bit_identical(cuda, n):
    """The FP64 blocked LU's trailing update on the tensor cores (DMMA) and on the FP64
    pipe give the same factors, pivots and info bit for bit, and both equal the oracle."""
    import torch

    import magma_b200 as mb
    import oracle
    from magma_b200 import testing as T
    lib = _lib.load()
    orig = _get(lib)
    batch = max(2, 3_000_000 // (n * n))
    A_np, _ = T.lu_uniform(batch, n, 1, seed=n)
    A_np[0, 7, :] = 0.0                      # a singular instance (zero column 8)
    res = {}
    try:
        for v in (0, 1):
            assert _set(lib, orig[:9] + [v] * 4 + orig[13:]) == 0
            A = torch.from_numpy(A_np).to(cuda)
            ipiv, info = mb.dgetrf_batched(A)
            torch.cuda.synchronize()
            res[v] = (A.cpu().numpy(), ipiv.cpu().numpy(), info.cpu().numpy())
    finally:
        _set(lib, orig)
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)
    O = A_np[:3].copy()
    oip, oinf = oracle.dgetrf_batched(O, n)
    assert np.array_equal(res[1][0][:3], O) and np.array_equal(res[1][1][:3], oip)
    assert np.array_equal(res[1][2][:3], oinf) and oinf[0] == 8


@pytest.mark.gpu
@pytest.mark.parametrize("n", [96, 160, 256])
def test_mixed_paths_per_order(cuda, n):
    """The tuning table's per-order switch between the tensor-core LU with its fused
    refinement and the CUDA-core FP32 LU with the separate refinement kernel: both meet
    the backward-error bound on the same systems."""
    import torch

    import magma_b200 as mb
    from magma_b200 import testing as T
    lib = _lib.load()
    orig = _get(lib)
    A_np, B_np, _ = T.svd_logrand(24, n, 1e2, 1e6, nrhs=4, seed=900 + n)
    try:
        for v in (0, 1):
            vals = list(orig)
            vals[13 + (n - 96) // 32] = v
            assert _set(lib, vals) == 0
            X, ipiv, it, info = mb.dsgesv_batched(torch.from_numpy(A_np).to(cuda), torch.from_numpy(B_np).to(cuda))
            assert T.backward_error(A_np, X.cpu().numpy(), B_np, n).max() <= 1e-14
            assert (it.cpu().numpy() >= 0).mean() >= 0.9 and not info.cpu().numpy().any()
    finally:
        _set(lib, orig)
