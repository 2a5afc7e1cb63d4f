"""Torch-facing wrappers over the C ABI.

Matrices are column-major, as in MAGMA: a batch of (m x n) matrices with
leading dimension ld is a CUDA tensor of shape (batch, n, ld) whose entry
[b, j, i] is A_b(i, j). The wrappers build MAGMA's device pointer arrays
(``ptr_array``), allocate the caller-owned outputs (ipiv, info) and call the
library on a queue that wraps the current torch stream. They raise on a
negative (argument-error) return code.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import MagmaNoTrans, MagmaTrans


class Queue:
    """A magma_queue_t wrapping a CUDA stream (torch's current stream by default)."""

    def __init__(self, stream: torch.cuda.Stream | None = None, device: int | None = None):
        self.lib = _lib.load()
        if device is None:
            device = torch.cuda.current_device()
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        q = C.c_void_p()
        self.lib.magma_queue_create_from_cuda_internal(device, C.c_void_p(self.stream.cuda_stream), None, None,
                                                       C.byref(q), b"Queue", b"api.py", 0)
        self.handle = q

    def sync(self) -> None:
        self.lib.magma_queue_sync_internal(self.handle, b"Queue.sync", b"api.py", 0)

    def reserve(self, nbytes: int) -> None:
        rc = self.lib.magma_queue_reserve_workspace(self.handle, nbytes)
        if rc != 0:
            raise MemoryError(f"magma_queue_reserve_workspace({nbytes}) failed: {rc}")

    def close(self) -> None:
        if self.handle:
            self.lib.magma_queue_destroy_internal(self.handle, b"Queue.close", b"api.py", 0)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_queues: dict[tuple[int, int], Queue] = {}


def default_queue() -> Queue:
    dev = torch.cuda.current_device()
    s = torch.cuda.current_stream(dev)
    key = (dev, s.cuda_stream)
    q = _default_queues.get(key)
    if q is None:
        q = Queue(s, dev)
        _default_queues[key] = q
    return q


def ptr_array(t: torch.Tensor) -> torch.Tensor:
    """Device array (int64) of per-instance base pointers of a batched tensor."""
    assert t.is_cuda
    n = t.shape[0]
    step = t.stride(0) * t.element_size()
    return t.data_ptr() + torch.arange(n, device=t.device, dtype=torch.int64) * step


def _vp(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def _check(rc: int, name: str) -> int:
    if rc < 0:
        raise ValueError(f"{name} returned {rc} (illegal argument {-rc})" if rc > -100
                         else f"{name} returned MAGMA error {rc}")
    return rc


def dgetrf_batched(A: torch.Tensor, m: int | None = None, queue: Queue | None = None):
    """LU with partial pivoting of each (m x n) instance of A (batch, n, lda), in place.

    Returns (ipiv (batch, min(m,n)) int32, 1-based; info (batch,) int32)."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    m = lda if m is None else m
    ipiv = torch.zeros((batch, max(1, min(m, n))), dtype=torch.int32, device=A.device)
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pP = ptr_array(A), ptr_array(ipiv)
    rc = q.lib.magma_dgetrf_batched(m, n, _vp(pA), lda, _vp(pP), _vp(info), batch, q.handle)
    _check(rc, "magma_dgetrf_batched")
    return ipiv, info


def dgetrs_batched(A: torch.Tensor, ipiv: torch.Tensor, B: torch.Tensor, trans: bool = False,
                   queue: Queue | None = None) -> None:
    """Solve op(A_i) X_i = B_i with the factors from dgetrf_batched; B (batch, nrhs, ldb) in place."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    # keep the pointer arrays referenced until the call is enqueued: a temporary
    # freed early would be handed to the next allocation by torch's caching allocator
    pA, pP, pB = ptr_array(A), ptr_array(ipiv), ptr_array(B)
    rc = q.lib.magma_dgetrs_batched(MagmaTrans if trans else MagmaNoTrans, n, nrhs, _vp(pA), lda,
                                    _vp(pP), _vp(pB), ldb, batch, q.handle)
    _check(rc, "magma_dgetrs_batched")


def dgesv_batched(A: torch.Tensor, B: torch.Tensor, queue: Queue | None = None):
    """Factor and solve each A_i X_i = B_i in place. Returns (ipiv, info)."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    ipiv = torch.zeros((batch, n), dtype=torch.int32, device=A.device)
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pP, pB = ptr_array(A), ptr_array(ipiv), ptr_array(B)
    rc = q.lib.magma_dgesv_batched(n, nrhs, _vp(pA), lda, _vp(pP), _vp(pB), ldb, _vp(info), batch, q.handle)
    _check(rc, "magma_dgesv_batched")
    return ipiv, info
