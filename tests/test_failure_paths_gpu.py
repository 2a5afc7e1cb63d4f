"""Failure paths, exercised without faulting the GPU.

* A queue whose workspace limit is below what a batched call needs makes the call
  return MAGMA_ERR_DEVICE_ALLOC (-113) before it enqueues anything, as the reference
  does when its per-call cudaMalloc fails (src/zgetrf_batched.cpp:172-194,
  src/zpotrf_vbatched.cpp:99,124); the same call succeeds once the limit is lifted.
* The request loop reports that code as the info of every request of the failed
  micro-batch, and serves later requests normally.
* The tensor-core LU's bounded completion wait: under the test hook the kernel issues
  no tensor-core work, so its wait runs out with nothing in flight; every instance
  must then come out of the FP64 fallback (iter -3) with the plain FP64 path's
  factors and pivots, bit for bit, and solutions at backward error <= 1e-14.
"""
import ctypes as C

import numpy as np
import pytest

from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
DEVICE_ALLOC = -113
NO_LIMIT = 2**64 - 1


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def test_workspace_limit_returns_device_alloc(cuda):
    import torch

    from magma_b200.api import Queue, VarBatch
    stream = torch.cuda.Stream(cuda)
    q = Queue(stream, 0)
    lib = q.lib
    vp = lambda t: C.c_void_p(t.data_ptr())
    # variable-size LU solve: the size bucketing needs queue workspace
    ns = np.array([5, 40, 77, 130, 9], np.int32)
    As = [T.lu_uniform(1, int(n), 1, seed=int(n))[0][0] for n in ns]
    Bs = [T.lu_uniform(1, int(n), 2, seed=int(n) + 1)[1][0] for n in ns]
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    nrhs = np.full(len(ns), 2, np.int32)
    dn, dr = gA.ints(ns), gA.ints(nrhs)
    piv = torch.zeros(len(ns), 130, dtype=torch.int32, device=cuda)
    pP = piv.data_ptr() + torch.arange(len(ns), device=cuda, dtype=torch.int64) * 130 * 4
    info = torch.full((len(ns) + 1,), 77, dtype=torch.int32, device=cuda)
    A0, B0 = gA.buf.clone(), gB.buf.clone()
    call = lambda: lib.magma_dgesv_vbatched(vp(dn), vp(dr), vp(gA.ptrs), vp(dn), vp(pP), vp(gB.ptrs), vp(dn),
                                            vp(info), len(ns), q.handle)
    assert lib.magma_b200_queue_set_workspace_limit(q.handle, 0) == 0
    assert call() == DEVICE_ALLOC
    q.sync()
    assert torch.equal(gA.buf, A0) and torch.equal(gB.buf, B0)      # nothing was enqueued
    assert (info == 77).all()
    # the mixed solve's workspace too
    A_np, B_np, _ = T.svd_logrand(3, 128, 1e2, 1e4, nrhs=2, seed=5)
    from magma_b200.api import ptr_array
    A, B = dev(A_np, cuda), dev(B_np, cuda)
    X = torch.zeros_like(B)
    it = torch.zeros(3, dtype=torch.int32, device=cuda)
    inf = torch.zeros(3, dtype=torch.int32, device=cuda)
    ip = torch.zeros(3, 128, dtype=torch.int32, device=cuda)
    pA, pB, pX, pI = ptr_array(A), ptr_array(B), ptr_array(X), ptr_array(ip)
    mixed = lambda: lib.magma_dsgesv_batched(128, 2, vp(pA), 128, vp(pI), vp(pB), 128, vp(pX), 128, vp(it),
                                             vp(inf), 3, q.handle)
    assert mixed() == DEVICE_ALLOC
    # lifted: both calls run
    assert lib.magma_b200_queue_set_workspace_limit(q.handle, NO_LIMIT) == 0
    assert call() == 0 and mixed() == 0
    q.sync()
    assert (info[:len(ns)] == 0).all()
    assert T.backward_error(A_np, X.cpu().numpy(), B_np, 128).max() <= 1e-14
    q.close()


def test_request_loop_reports_device_alloc(cuda):
    from magma_b200 import serve
    reqs = serve.make_requests(8, seed=21, n_lo=16, n_hi=200)
    with serve.Server(1 << 28, streams=1, max_batch=64) as sv:
        sv.set_workspace_limit(0)
        for i, r in enumerate(reqs):
            sv.submit(r.kind, r.A, r.B, r.X, i)
        sv.drain()
        tags, infos, _, _ = sv.poll()
        assert sorted(tags.tolist()) == list(range(8))
        assert (infos == DEVICE_ALLOC).all(), infos
        sv.set_workspace_limit(NO_LIMIT)
        for i, r in enumerate(reqs):
            sv.submit(r.kind, r.A, r.B, r.X, 100 + i)
        sv.drain()
        tags, infos, _, _ = sv.poll()
        assert sorted(tags.tolist()) == list(range(100, 108)) and not infos.any()
    for r in reqs:
        assert serve.backward_error(r) <= 1e-14


def test_tensor_core_wait_timeout_falls_back_to_fp64(cuda):
    import magma_b200 as mb
    from magma_b200 import _lib
    lib = _lib.load()
    n, batch = 256, 20   # an order the built-in table runs on the tensor-core LU
    A_np, B_np, _ = T.svd_logrand(batch, n, 1e2, 1e6, nrhs=4, seed=31)
    lib.magma_b200_debug_tc_wait_limit(100000)
    try:
        A = dev(A_np, cuda)
        X, ipiv, it, info = mb.dsgesv_batched(A, dev(B_np, cuda))
        it, info = it.cpu().numpy(), info.cpu().numpy()
    finally:
        lib.magma_b200_debug_tc_wait_limit(0)
    assert (it == -3).all(), it
    assert not info.any()
    A64, B64 = dev(A_np, cuda), dev(B_np, cuda)
    p64, i64 = mb.dgesv_batched(A64, B64)
    assert np.array_equal(A.cpu().numpy(), A64.cpu().numpy())
    assert np.array_equal(ipiv.cpu().numpy(), p64.cpu().numpy())
    assert np.array_equal(X.cpu().numpy(), B64.cpu().numpy())
    assert T.backward_error(A_np, X.cpu().numpy(), B_np, n).max() <= 1e-14
    # normal operation afterwards: the tensor-core path refines again
    X2, _, it2, _ = mb.dsgesv_batched(dev(A_np, cuda), dev(B_np, cuda))
    assert (it2.cpu().numpy() >= 0).mean() >= 0.9
    assert T.backward_error(A_np, X2.cpu().numpy(), B_np, n).max() <= 1e-14
