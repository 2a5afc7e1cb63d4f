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
from ._lib import MagmaLeft, MagmaNonUnit, MagmaNoTrans, MagmaRight, MagmaTrans, MagmaUnit


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
    if not t.is_cuda:
        raise ValueError("ptr_array needs a CUDA tensor (the library takes device pointer arrays)")
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


# ---------------------------------------------------------------------------- Cholesky
from ._lib import MagmaLower, MagmaUpper  # noqa: E402


def _uplo(upper: bool) -> int:
    return MagmaUpper if upper else MagmaLower


def dpotrf_batched(A: torch.Tensor, upper: bool = False, queue: Queue | None = None) -> torch.Tensor:
    """Cholesky of each instance of A (batch, n, lda) in place. Returns info (batch,)."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA = ptr_array(A)
    _check(q.lib.magma_dpotrf_batched(_uplo(upper), n, _vp(pA), lda, _vp(info), batch, q.handle),
           "magma_dpotrf_batched")
    return info


def dpotrs_batched(A: torch.Tensor, B: torch.Tensor, upper: bool = False, queue: Queue | None = None) -> None:
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dpotrs_batched(_uplo(upper), n, nrhs, _vp(pA), lda, _vp(pB), ldb, batch, q.handle),
           "magma_dpotrs_batched")


def dposv_batched(A: torch.Tensor, B: torch.Tensor, upper: bool = False, queue: Queue | None = None) -> torch.Tensor:
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dposv_batched(_uplo(upper), n, nrhs, _vp(pA), lda, _vp(pB), ldb, _vp(info), batch, q.handle),
           "magma_dposv_batched")
    return info


class VarBatch:
    """Variable-size batch packed into one device buffer, with MAGMA's pointer
    array and per-instance size arrays (batchCount+1 entries, last one scratch).

    ``mats`` are column-major host arrays of shape (cols_i, ld_i)."""

    def __init__(self, mats, device, dtype=torch.float64, align: int = 32):
        import numpy as np

        self.batch = len(mats)
        self.shapes = [tuple(m.shape) for m in mats]
        esz = torch.tensor([], dtype=dtype).element_size()
        step = max(1, align // esz)
        sizes = [((m.size + step - 1) // step) * step for m in mats]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if mats else np.zeros(0, np.int64)
        total = int(sum(sizes)) if mats else 1
        flat = np.zeros(max(total, 1), dtype=np.float64 if dtype == torch.float64 else np.float32)
        self.dtype = dtype
        for m, o in zip(mats, self.offsets):
            flat[o:o + m.size] = m.reshape(-1)
        self.buf = torch.from_numpy(flat).to(device)
        self.ptrs = self.buf.data_ptr() + torch.from_numpy(self.offsets * esz).to(device)
        self.device = device

    def ints(self, values) -> torch.Tensor:
        """Device int32 array of batch+1 entries (the extra slot is scratch)."""
        import numpy as np

        v = np.zeros(self.batch + 1, np.int32)
        v[:self.batch] = values
        return torch.from_numpy(v).to(self.device)

    def unpack(self):
        flat = self.buf.cpu().numpy()
        return [flat[o:o + s[0] * s[1]].reshape(s).copy() for o, s in zip(self.offsets, self.shapes)]


def dposv_vbatched(A: VarBatch, B: VarBatch | None, n, nrhs=None, lda=None, ldb=None, upper=False,
                   factor=True, solve=True, max_sizes=None, queue: Queue | None = None):
    """Variable-size potrf / potrs / posv through the C ABI. Returns info (device) or None for potrs.

    max_sizes=(max_n, max_nrhs) selects the _max_nocheck entry points."""
    q = queue or default_queue()
    batch = A.batch
    dn = A.ints(n)
    dlda = A.ints(lda if lda is not None else [s[1] for s in A.shapes])
    dB = B.ptrs if B is not None else None
    dnr = A.ints(nrhs) if nrhs is not None else None
    dldb = A.ints(ldb if ldb is not None else [s[1] for s in B.shapes]) if B is not None else None
    info = torch.empty(batch + 1, dtype=torch.int32, device=A.device)
    L = q.lib
    u = _uplo(upper)
    if factor and not solve:
        if max_sizes:
            rc = L.magma_dpotrf_vbatched_max_nocheck(u, _vp(dn), _vp(A.ptrs), _vp(dlda), _vp(info), batch,
                                                     max_sizes[0], q.handle)
        else:
            rc = L.magma_dpotrf_vbatched(u, _vp(dn), _vp(A.ptrs), _vp(dlda), _vp(info), batch, q.handle)
        _check(rc, "magma_dpotrf_vbatched")
        return info[:batch]
    if solve and not factor:
        if max_sizes:
            rc = L.magma_dpotrs_vbatched_max_nocheck(u, _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dlda), _vp(dB),
                                                     _vp(dldb), batch, max_sizes[0], max_sizes[1], q.handle)
        else:
            rc = L.magma_dpotrs_vbatched(u, _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dlda), _vp(dB), _vp(dldb), batch,
                                         q.handle)
        _check(rc, "magma_dpotrs_vbatched")
        return None
    if max_sizes:
        rc = L.magma_dposv_vbatched_max_nocheck(u, _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dlda), _vp(dB), _vp(dldb),
                                                _vp(info), batch, max_sizes[0], max_sizes[1], q.handle)
    else:
        rc = L.magma_dposv_vbatched(u, _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dlda), _vp(dB), _vp(dldb), _vp(info),
                                    batch, q.handle)
    _check(rc, "magma_dposv_vbatched")
    return info[:batch]


# -------------------------------------------------------------------- mixed precision
def dsgesv_batched(A: torch.Tensor, B: torch.Tensor, queue: Queue | None = None):
    """Mixed-precision solve A_i X_i = B_i (FP32 LU, FP64 refinement, FP64 fallback).

    Returns (X, ipiv, iter, info); A is left unchanged unless iter < 0."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    X = torch.empty((batch, nrhs, n), dtype=torch.float64, device=A.device)
    ipiv = torch.zeros((batch, n), dtype=torch.int32, device=A.device)
    it = torch.empty(batch, dtype=torch.int32, device=A.device)
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pP, pB, pX = ptr_array(A), ptr_array(ipiv), ptr_array(B), ptr_array(X)
    _check(q.lib.magma_dsgesv_batched(n, nrhs, _vp(pA), lda, _vp(pP), _vp(pB), ldb, _vp(pX), n, _vp(it), _vp(info),
                                      batch, q.handle), "magma_dsgesv_batched")
    return X, ipiv, it, info


class _HostPipeline:
    """Batched solve of systems that live in pinned host memory, with the transfers
    pipelined against the solves: a binding of the library's magma_b200_host_solver
    (include/magma_b200.h).

    The batch is cut into `chunks` slices. All slices' uploads are queued on one copy
    stream, back to back, so the host-to-device link never idles; slice c is solved on the
    queue's stream as soon as its upload has landed, and its results go back to the host on
    a second copy stream while later slices are still uploading or solving. Every kernel
    works instance by instance, so the results equal those of one call over the whole batch.

    A call is asynchronous: it returns once everything is queued, and the queue's stream
    waits for the last read-back, so a stream synchronize (or an event recorded on that
    stream) covers the whole transfer-solve-transfer sequence. Device staging buffers,
    streams, events and pointer arrays are allocated once, by the library, at construction."""

    _kind = 0

    def __init__(self, batch: int, n: int, nrhs: int, chunks: int, queue: Queue | None, lda: int | None,
                 ldb: int | None):
        if batch < 1 or n < 1 or nrhs < 1 or chunks < 1:
            raise ValueError("batch, n, nrhs and chunks must be positive")
        self.q = queue or default_queue()
        self.batch, self.n, self.nrhs = batch, n, nrhs
        self.lda, self.ldb = lda or n, ldb or n
        if self.lda < n or self.ldb < n:
            raise ValueError("lda and ldb must be at least n")
        h = C.c_void_p()
        _check(self.q.lib.magma_b200_host_solver_create(self._kind, batch, n, nrhs, self.lda, self.ldb, chunks,
                                                        self.q.handle, C.byref(h)), "magma_b200_host_solver_create")
        self.h = h
        starts = []
        c = 0
        while True:
            st = self.q.lib.magma_b200_host_solver_chunk_start(h, c)
            if st < 0:
                break
            starts.append(st)
            c += 1
        self.bounds = list(zip(starts[:-1], starts[1:]))

    def _shapes(self):
        raise NotImplementedError

    def _run(self, hA, hB, hX, hI, hInfo) -> None:
        shapes = self._shapes()
        for t, (shape, dtype), name in zip((hA, hB, hX, hI, hInfo), shapes, ("hA", "hB", "hX", "hI", "hInfo")):
            if t.is_cuda or not t.is_pinned():
                raise ValueError(f"{type(self).__name__} takes pinned host tensors ({name})")
            if tuple(t.shape) != shape or t.dtype != dtype or not t.is_contiguous():
                raise ValueError(f"{name} of shape {tuple(t.shape)} ({t.dtype}) expected {shape} ({dtype}), contiguous")
        _check(self.q.lib.magma_b200_host_solve(self.h, _vp(hA), _vp(hB), _vp(hX), _vp(hI), _vp(hInfo)),
               "magma_b200_host_solve")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.q.lib.magma_b200_host_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostDsgesv(_HostPipeline):
    """magma_dsgesv_batched (FP32 LU, FP64 refinement, FP64 fallback) on systems in pinned
    host memory, uploads and read-backs overlapped with the solves chunk by chunk."""

    _kind = 0   # MAGMA_B200_HOST_DSGESV

    def __init__(self, batch: int, n: int, nrhs: int, chunks: int = 8, queue: Queue | None = None,
                 lda: int | None = None, ldb: int | None = None):
        super().__init__(batch, n, nrhs, chunks, queue, lda, ldb)

    def _shapes(self):
        b, n, r = self.batch, self.n, self.nrhs
        f64, i32 = torch.float64, torch.int32
        return [((b, n, self.lda), f64), ((b, r, self.ldb), f64), ((b, r, n), f64), ((b,), i32), ((b,), i32)]

    def __call__(self, hA: torch.Tensor, hB: torch.Tensor, hX: torch.Tensor, hIter: torch.Tensor,
                 hInfo: torch.Tensor) -> None:
        """hA (batch, n, lda) and hB (batch, nrhs, ldb) in, hX (batch, nrhs, n), hIter and
        hInfo (batch, int32) out; all pinned host tensors."""
        self._run(hA, hB, hX, hIter, hInfo)


class HostDgesv(_HostPipeline):
    """magma_dgesv_batched (FP64 LU with partial pivoting + solve) on systems in pinned host
    memory, uploads and read-backs overlapped with the solves chunk by chunk."""

    _kind = 1   # MAGMA_B200_HOST_DGESV

    def __init__(self, batch: int, n: int, nrhs: int, chunks: int = 4, queue: Queue | None = None,
                 lda: int | None = None, ldb: int | None = None):
        super().__init__(batch, n, nrhs, chunks, queue, lda, ldb)

    def _shapes(self):
        b, n, r = self.batch, self.n, self.nrhs
        f64, i32 = torch.float64, torch.int32
        return [((b, n, self.lda), f64), ((b, r, self.ldb), f64), ((b, r, self.ldb), f64), ((b, n), i32), ((b,), i32)]

    def __call__(self, hA: torch.Tensor, hB: torch.Tensor, hX: torch.Tensor, hIpiv: torch.Tensor,
                 hInfo: torch.Tensor) -> None:
        """hA (batch, n, lda) and hB (batch, nrhs, ldb) in; hX (batch, nrhs, ldb) = the
        solutions, hIpiv (batch, n) and hInfo (batch,) int32 out; all pinned host tensors."""
        self._run(hA, hB, hX, hIpiv, hInfo)


# ------------------------------------------------------------------------------- GEMM
def _trans(t: bool) -> int:
    return MagmaTrans if t else MagmaNoTrans


def gemm_batched(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, m: int, n: int, k: int, alpha=1.0, beta=0.0,
                 transA=False, transB=False, queue: Queue | None = None) -> None:
    """C_i = alpha op(A_i) op(B_i) + beta C_i for column-major batches (batch, cols, ld), in place."""
    q = queue or default_queue()
    batch = C.shape[0]
    pre = "d" if C.dtype == torch.float64 else "s"
    fn = getattr(q.lib, f"magmablas_{pre}gemm_batched")
    pA, pB, pC = ptr_array(A), ptr_array(B), ptr_array(C)
    fn(_trans(transA), _trans(transB), m, n, k, alpha, _vp(pA), A.shape[2], _vp(pB), B.shape[2], beta, _vp(pC),
       C.shape[2], batch, q.handle)


def gemm_vbatched(A: "VarBatch", B: "VarBatch", C: "VarBatch", m, n, k, lda, ldb, ldc, alpha=1.0, beta=0.0,
                  transA=False, transB=False, max_sizes=None, queue: Queue | None = None) -> None:
    """Variable-size GEMM through magmablas_{d,s}gemm_vbatched (or _max_nocheck when max_sizes is given)."""
    q = queue or default_queue()
    pre = "d" if C.buf.dtype == torch.float64 else "s"
    dm, dn, dk = C.ints(m), C.ints(n), C.ints(k)
    dla, dlb, dlc = C.ints(lda), C.ints(ldb), C.ints(ldc)
    args = [_trans(transA), _trans(transB), _vp(dm), _vp(dn), _vp(dk), alpha, _vp(A.ptrs), _vp(dla), _vp(B.ptrs),
            _vp(dlb), beta, _vp(C.ptrs), _vp(dlc), C.batch]
    if max_sizes:
        getattr(q.lib, f"magmablas_{pre}gemm_vbatched_max_nocheck")(*args, *max_sizes, q.handle)
    else:
        getattr(q.lib, f"magmablas_{pre}gemm_vbatched")(*args, q.handle)


# --------------------------------------------------------------- variable-size LU
def dgesv_vbatched(A: "VarBatch", B: "VarBatch | None", n, nrhs=None, lda=None, ldb=None, m=None, factor=True,
                   solve=True, trans=False, ipiv: torch.Tensor | None = None, max_sizes=None,
                   queue: Queue | None = None):
    """Variable-size getrf / getrs / gesv through the C ABI.

    Returns (ipiv (batch, max) int32 device tensor, info device tensor or None). For getrs
    pass the ipiv returned by the factorisation. max_sizes selects the _max_nocheck forms
    ((max_m, max_n) for getrf, (max_n, max_nrhs) otherwise)."""
    import numpy as np

    q = queue or default_queue()
    L = q.lib
    batch = A.batch
    n = np.asarray(n, np.int32)
    m = n if m is None else np.asarray(m, np.int32)
    lda = [s[1] for s in A.shapes] if lda is None else lda
    dm, dn, dla = A.ints(m), A.ints(n), A.ints(lda)
    width = int(max(1, np.minimum(m, n).max() if batch else 1))
    if ipiv is None:
        ipiv = torch.zeros((batch, width), dtype=torch.int32, device=A.device)
    pP = ptr_array(ipiv)
    info = torch.empty(batch + 1, dtype=torch.int32, device=A.device)
    if factor and not solve:
        if max_sizes:
            rc = L.magma_dgetrf_vbatched_max_nocheck(_vp(dm), _vp(dn), _vp(A.ptrs), _vp(dla), _vp(pP), _vp(info),
                                                     batch, max_sizes[0], max_sizes[1], q.handle)
        else:
            rc = L.magma_dgetrf_vbatched(_vp(dm), _vp(dn), _vp(A.ptrs), _vp(dla), _vp(pP), _vp(info), batch, q.handle)
        _check(rc, "magma_dgetrf_vbatched")
        return ipiv, info[:batch]
    dnr = A.ints(nrhs)
    dlb = A.ints([s[1] for s in B.shapes] if ldb is None else ldb)
    if solve and not factor:
        if max_sizes:
            rc = L.magma_dgetrs_vbatched_max_nocheck(_trans(trans), _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dla), _vp(pP),
                                                     _vp(B.ptrs), _vp(dlb), batch, max_sizes[0], max_sizes[1],
                                                     q.handle)
        else:
            rc = L.magma_dgetrs_vbatched(_trans(trans), _vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dla), _vp(pP),
                                         _vp(B.ptrs), _vp(dlb), batch, q.handle)
        _check(rc, "magma_dgetrs_vbatched")
        return ipiv, None
    if max_sizes:
        rc = L.magma_dgesv_vbatched_max_nocheck(_vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dla), _vp(pP), _vp(B.ptrs),
                                                _vp(dlb), _vp(info), batch, max_sizes[0], max_sizes[1], q.handle)
    else:
        rc = L.magma_dgesv_vbatched(_vp(dn), _vp(dnr), _vp(A.ptrs), _vp(dla), _vp(pP), _vp(B.ptrs), _vp(dlb),
                                    _vp(info), batch, q.handle)
    _check(rc, "magma_dgesv_vbatched")
    return ipiv, info[:batch]


def dsposv_vbatched(A: "VarBatch", B: "VarBatch", n, nrhs, lda=None, ldb=None, max_sizes=None,
                    queue: Queue | None = None):
    """Variable-size mixed-precision Cholesky solve (magma_dsposv_vbatched, Lower).

    Returns (X as a VarBatch shaped like B, iter, info); the single-precision
    workspaces (n_i*(n_i+nrhs_i) floats each) are allocated here."""
    import numpy as np

    q = queue or default_queue()
    batch = A.batch
    X = VarBatch([np.zeros(s) for s in B.shapes], A.device)
    nn = np.asarray(n, np.int64)
    rr = np.asarray(nrhs, np.int64)
    words = ((nn * (nn + rr) + 7) // 8) * 8
    offs = np.concatenate([[0], np.cumsum(words)[:-1]]) if batch else np.zeros(0, np.int64)
    S = torch.empty(max(int(words.sum()), 1), dtype=torch.float32, device=A.device)
    Sp = S.data_ptr() + torch.from_numpy(offs * 4).to(A.device)
    dn, dr = A.ints(n), A.ints(nrhs)
    dla = A.ints(lda if lda is not None else [s[1] for s in A.shapes])
    dlb = A.ints(ldb if ldb is not None else [s[1] for s in B.shapes])
    dlx = A.ints([s[1] for s in X.shapes])
    it = torch.empty(batch + 1, dtype=torch.int32, device=A.device)
    info = torch.empty(batch + 1, dtype=torch.int32, device=A.device)
    args = [MagmaLower, _vp(dn), _vp(dr), _vp(A.ptrs), _vp(dla), _vp(B.ptrs), _vp(dlb), _vp(X.ptrs), _vp(dlx),
            _vp(Sp), _vp(it), _vp(info), batch]
    if max_sizes:
        rc = q.lib.magma_dsposv_vbatched_max_nocheck(*args, max_sizes[0], max_sizes[1], q.handle)
    else:
        rc = q.lib.magma_dsposv_vbatched(*args, q.handle)
    _check(rc, "magma_dsposv_vbatched")
    q.sync()
    del S
    return X, it[:batch], info[:batch]


def dgetri_outofplace_batched(LU: torch.Tensor, ipiv: torch.Tensor, queue: Queue | None = None):
    """inv(A_i) from getrf factors (column-major batch (batch, n, ld)). Returns (invA, info)."""
    q = queue or default_queue()
    batch, n, lda = LU.shape
    inv = torch.empty((batch, n, n), dtype=torch.float64, device=LU.device)
    info = torch.empty(batch, dtype=torch.int32, device=LU.device)
    pA, pP, pI = ptr_array(LU), ptr_array(ipiv), ptr_array(inv)
    _check(q.lib.magma_dgetri_outofplace_batched(n, _vp(pA), lda, _vp(pP), _vp(pI), n, _vp(info), batch, q.handle),
           "magma_dgetri_outofplace_batched")
    return inv, info


def dgetrf_nopiv_batched(A: torch.Tensor, m: int | None = None, queue: Queue | None = None) -> torch.Tensor:
    """LU without pivoting of each instance of A (batch, n, lda), in place. Returns info."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    m = lda if m is None else m
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA = ptr_array(A)
    _check(q.lib.magma_dgetrf_nopiv_batched(m, n, _vp(pA), lda, _vp(info), batch, q.handle),
           "magma_dgetrf_nopiv_batched")
    return info


def dgetrs_nopiv_batched(A: torch.Tensor, B: torch.Tensor, trans: bool = False, queue: Queue | None = None) -> None:
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dgetrs_nopiv_batched(_trans(trans), n, nrhs, _vp(pA), lda, _vp(pB), ldb, None, batch,
                                            q.handle), "magma_dgetrs_nopiv_batched")


def dgesv_nopiv_batched(A: torch.Tensor, B: torch.Tensor, queue: Queue | None = None) -> torch.Tensor:
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dgesv_nopiv_batched(n, nrhs, _vp(pA), lda, _vp(pB), ldb, _vp(info), batch, q.handle),
           "magma_dgesv_nopiv_batched")
    return info


def dgerbt_batched(A: torch.Tensor, B: torch.Tensor, U=None, V=None, queue: Queue | None = None):
    """A_i <- U^T A_i V, B_i <- U^T B_i (in place). Without U, V a butterfly is generated;
    returns the (U, V) numpy vectors used (2n entries each)."""
    import numpy as np

    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    gen = U is None
    hu = np.zeros(2 * n) if gen else np.ascontiguousarray(U, dtype=np.float64).copy()
    hv = np.zeros(2 * n) if gen else np.ascontiguousarray(V, dtype=np.float64).copy()
    info = C.c_int(0)
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dgerbt_batched(1 if gen else 0, n, nrhs, _vp(pA), lda, _vp(pB), ldb, hu.ctypes.data,
                                      hv.ctypes.data, C.byref(info), batch, q.handle), "magma_dgerbt_batched")
    q.sync()
    return hu, hv


def dgesv_rbt_batched(A: torch.Tensor, B: torch.Tensor, queue: Queue | None = None) -> torch.Tensor:
    q = queue or default_queue()
    batch, n, lda = A.shape
    _, nrhs, ldb = B.shape
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pB = ptr_array(A), ptr_array(B)
    _check(q.lib.magma_dgesv_rbt_batched(n, nrhs, _vp(pA), lda, _vp(pB), ldb, _vp(info), batch, q.handle),
           "magma_dgesv_rbt_batched")
    return info


def dgeqrf_batched(A: torch.Tensor, m: int | None = None, queue: Queue | None = None) -> torch.Tensor:
    """Householder QR of each (m x n) instance of A (batch, n, lda), in place. Returns tau."""
    q = queue or default_queue()
    batch, n, lda = A.shape
    m = lda if m is None else m
    tau = torch.zeros((batch, max(1, min(m, n))), dtype=torch.float64, device=A.device)
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    pA, pT = ptr_array(A), ptr_array(tau)
    _check(q.lib.magma_dgeqrf_batched(m, n, _vp(pA), lda, _vp(pT), _vp(info), batch, q.handle),
           "magma_dgeqrf_batched")
    return tau


def syrk_vbatched(A: "VarBatch", C: "VarBatch", n, k, lda, ldc, alpha=1.0, beta=0.0, lower=True, trans=False,
                  max_sizes=None, checked=True, queue: Queue | None = None) -> None:
    """Variable-size SYRK through magmablas_{d,s}syrk_vbatched{,_max_nocheck,_nocheck}."""
    q = queue or default_queue()
    pre = "d" if C.buf.dtype == torch.float64 else "s"
    dn, dk, dla, dlc = C.ints(n), C.ints(k), C.ints(lda), C.ints(ldc)
    args = [MagmaLower if lower else MagmaUpper, _trans(trans), _vp(dn), _vp(dk), alpha, _vp(A.ptrs), _vp(dla),
            beta, _vp(C.ptrs), _vp(dlc), C.batch]
    if max_sizes:
        getattr(q.lib, f"magmablas_{pre}syrk_vbatched_max_nocheck")(*args, *max_sizes, q.handle)
    elif checked:
        getattr(q.lib, f"magmablas_{pre}syrk_vbatched")(*args, q.handle)
    else:
        getattr(q.lib, f"magmablas_{pre}syrk_vbatched_nocheck")(*args, q.handle)


def tri_vbatched(op: str, A: "VarBatch", B: "VarBatch", m, n, lda, ldb, alpha=1.0, left=True, lower=True,
                 trans=False, unit=False, max_sizes=None, checked=True, queue: Queue | None = None) -> None:
    """Variable-size TRSM (op "trsm") or TRMM (op "trmm") through magmablas_{d,s}{op}_vbatched*."""
    q = queue or default_queue()
    pre = "d" if B.buf.dtype == torch.float64 else "s"
    dm, dn, dla, dlb = B.ints(m), B.ints(n), B.ints(lda), B.ints(ldb)
    args = [MagmaLeft if left else MagmaRight, MagmaLower if lower else MagmaUpper, _trans(trans),
            MagmaUnit if unit else MagmaNonUnit, _vp(dm), _vp(dn), alpha, _vp(A.ptrs), _vp(dla), _vp(B.ptrs),
            _vp(dlb), B.batch]
    if max_sizes:
        getattr(q.lib, f"magmablas_{pre}{op}_vbatched_max_nocheck")(*args, *max_sizes, q.handle)
    elif checked:
        getattr(q.lib, f"magmablas_{pre}{op}_vbatched")(*args, q.handle)
    else:
        getattr(q.lib, f"magmablas_{pre}{op}_vbatched_nocheck")(*args, q.handle)
