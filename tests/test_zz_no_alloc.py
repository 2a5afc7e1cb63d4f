"""GPU test of magma_dpotrf_vbatched_max_nocheck_noalloc, the variable-size
Cholesky entry point that allocates no device memory (for callers that cannot
allocate: graph capture in progress, fixed memory budgets, allocator
callbacks). Its scratch is a static device array inside the library.

It is called twice in a row through the C ABI, on two different batches, and
each result must be bit-identical (factors and info) to the regular
allocating entry point magma_dpotrf_vbatched_max_nocheck on the same input;
a batch above the static limit must be refused with -6 and leave the data
untouched. The file is named to run last in the suite."""
import numpy as np
import pytest

from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def _batch(count, nmax, seed):
    u = T.uniform01(seed, 11, count)
    a, b = 1.0, nmax ** -0.5
    ns = np.clip(np.round((a - u * (a - b)) ** -2), 1, nmax).astype(np.int32)
    mats = []
    for i, n in enumerate(ns):
        M = np.zeros((n, n))
        M[:, :] = T.spd_gram(int(n), seed, i)
        if i % 97 == 5:
            M[n // 2, n // 2] = -1.0          # a few instances are not positive definite
        mats.append(M)
    return ns, mats


def _run(entry, ns, mats, cuda):
    import torch

    from magma_b200.api import VarBatch, _vp, default_queue
    q = default_queue()
    A = VarBatch(mats, cuda)
    dn, dl = A.ints(ns), A.ints(ns)
    info = torch.full((len(ns) + 1,), -99, dtype=torch.int32, device=cuda)
    rc = getattr(q.lib, entry)(122, _vp(dn), _vp(A.ptrs), _vp(dl), _vp(info), len(ns), int(ns.max()), q.handle)
    torch.cuda.synchronize()
    return rc, A.unpack(), info[:len(ns)].cpu().numpy()


def test_noalloc_matches_allocating_entry_twice(cuda):
    for call, (count, nmax, seed) in enumerate([(3000, 300, 41), (1200, 700, 42)]):
        ns, mats = _batch(count, nmax, seed)
        rc0, ref, ref_info = _run("magma_dpotrf_vbatched_max_nocheck", ns, mats, cuda)
        rc1, got, got_info = _run("magma_dpotrf_vbatched_max_nocheck_noalloc", ns, mats, cuda)
        assert rc0 == 0 and rc1 == 0, (call, rc0, rc1)
        assert np.array_equal(got_info, ref_info), call
        assert (ref_info != 0).any() and (ref_info == 0).any()
        for i, n in enumerate(ns):
            assert np.array_equal(np.tril(got[i].T), np.tril(ref[i].T)), (call, i, n)


def test_noalloc_leaves_device_memory_unchanged(cuda):
    """After one warm call (which loads the kernels), a call changes the device's free
    memory by nothing: it allocates no device memory of its own."""
    import torch

    from magma_b200.api import VarBatch, _vp, default_queue
    q = default_queue()
    ns, mats = _batch(800, 400, 43)
    A = VarBatch(mats, cuda)
    dn = A.ints(ns)
    info = torch.zeros(len(ns) + 1, dtype=torch.int32, device=cuda)
    call = lambda: q.lib.magma_dpotrf_vbatched_max_nocheck_noalloc(122, _vp(dn), _vp(A.ptrs), _vp(dn), _vp(info),
                                                                   len(ns), int(ns.max()), q.handle)
    assert call() == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    assert call() == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free0


def test_noalloc_rejects_oversized_batch(cuda, capfd):
    import torch

    from magma_b200.api import _vp, default_queue
    q = default_queue()
    count = 65537
    dn = torch.ones(count + 1, dtype=torch.int32, device=cuda)
    buf = torch.full((count,), 4.0, dtype=torch.float64, device=cuda)
    ptrs = buf.data_ptr() + torch.arange(count, device=cuda, dtype=torch.int64) * 8
    info = torch.full((count + 1,), -99, dtype=torch.int32, device=cuda)
    rc = q.lib.magma_dpotrf_vbatched_max_nocheck_noalloc(122, _vp(dn), _vp(ptrs), _vp(dn), _vp(info), count, 1,
                                                         q.handle)
    torch.cuda.synchronize()
    assert rc == -6
    assert "exceeds" in capfd.readouterr().err
    assert (buf == 4.0).all() and (info == -99).all()
