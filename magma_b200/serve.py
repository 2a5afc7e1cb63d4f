"""Python driver of the request loop in libmagma_b200 (include/magma_b200_serve.h).

``Server`` wraps the C ABI. ``run_load`` replays an open-loop request stream
against it: Poisson arrivals at a given rate, 70% LU / 30% Cholesky requests,
n log-uniform in [8, 1024], RHS count uniform in {1..16}; LU matrices i.i.d.
uniform[-1, 1], Cholesky matrices G G^T + n I with G N(0, 1), right-hand sides
N(0, 1). Latency is measured from the request's scheduled arrival to the moment
its result is visible in host memory (both on the monotonic clock the library's
steady_clock uses), so a driver that falls behind its schedule is charged for it.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib

SOLVE_LU, SOLVE_CHOLESKY = 0, 1


class Server:
    """Owns one magma_b200_server (device arena, streams, worker threads)."""

    def __init__(self, budget_bytes: int, streams: int = 4, max_batch: int = 512, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.magma_b200_server_create(device, budget_bytes, streams, max_batch, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"magma_b200_server_create failed: {rc} ({self.lib.magma_strerror(rc).decode()})")
        self.h = h

    def submit(self, kind: int, A: np.ndarray, B: np.ndarray, X: np.ndarray, tag: int) -> None:
        """A (n x n), B and X (n x nrhs) are column-major float64 host arrays (Fortran order)
        that must stay alive until the request completes."""
        n, nrhs = A.shape[0], B.shape[1]
        rc = self.lib.magma_b200_server_submit(self.h, kind, n, nrhs, A.ctypes.data, n, B.ctypes.data, n,
                                               X.ctypes.data, n, tag)
        if rc != 0:
            raise ValueError(f"magma_b200_server_submit rejected request {tag}: {rc}")

    def poll(self, max_items: int = 4096):
        tags = np.empty(max_items, np.int64)
        infos = np.empty(max_items, np.int32)
        ts = np.empty(max_items, np.int64)
        td = np.empty(max_items, np.int64)
        k = self.lib.magma_b200_server_poll(self.h, tags.ctypes.data, infos.ctypes.data, ts.ctypes.data,
                                            td.ctypes.data, max_items)
        return tags[:k], infos[:k], ts[:k], td[:k]

    def drain(self) -> None:
        self.lib.magma_b200_server_drain(self.h)

    def set_workspace_limit(self, nbytes: int) -> None:
        """Caps each stream queue's device workspace (magma_b200_server_set_workspace_limit)."""
        self.lib.magma_b200_server_set_workspace_limit(self.h, nbytes)

    def stats(self) -> dict:
        v = [C.c_longlong() for _ in range(4)]
        self.lib.magma_b200_server_stats(self.h, *[C.byref(x) for x in v])
        return dict(zip(("submitted", "completed", "batches", "peak_bytes"), (x.value for x in v)))

    def close(self) -> None:
        if self.h:
            self.lib.magma_b200_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class Request:
    kind: int
    A: np.ndarray    # Fortran-ordered n x n
    B: np.ndarray    # Fortran-ordered n x nrhs
    X: np.ndarray    # result, Fortran-ordered n x nrhs
    host: object = None   # the pinned buffer the three arrays live in


class HostArena:
    """One page-locked host buffer carved into float64 Fortran-ordered arrays, so that
    the library's host<->device copies of request data are asynchronous."""

    def __init__(self, n_doubles: int):
        import torch
        self._t = torch.empty(max(n_doubles, 1), dtype=torch.float64, pin_memory=torch.cuda.is_available())
        self.buf = self._t.numpy()
        self.used = 0

    def take(self, rows: int, cols: int) -> np.ndarray:
        k = rows * cols
        k_al = (k + 31) & ~31          # 256-byte aligned carve-outs
        a = self.buf[self.used:self.used + k].reshape(cols, rows).T
        self.used += k_al
        return a


def make_requests(count: int, seed: int, n_lo: int = 8, n_hi: int = 1024, nrhs_hi: int = 16,
                  lu_share: float = 0.7) -> list[Request]:
    """The request mix, generated deterministically from `seed` into pinned host memory."""
    rng = np.random.default_rng(seed)
    kinds = np.where(rng.random(count) < lu_share, SOLVE_LU, SOLVE_CHOLESKY)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi + 1), count)).astype(np.int64).clip(n_lo, n_hi)
    nrhs = rng.integers(1, nrhs_hi + 1, count)
    total = int(sum(((n * n + 31) & ~31) + 2 * ((n * r + 31) & ~31) for n, r in zip(ns, nrhs)))
    arena = HostArena(total)
    reqs = []
    for i, (k, n, r) in enumerate(zip(kinds, ns, nrhs)):
        n, r = int(n), int(r)
        A, B, X = arena.take(n, n), arena.take(n, r), arena.take(n, r)
        sub = np.random.default_rng([seed, i])
        if k == SOLVE_LU:
            A[:] = sub.uniform(-1.0, 1.0, (n, n))
        else:
            G = sub.standard_normal((n, n))
            A[:] = G @ G.T + n * np.eye(n)
        B[:] = sub.standard_normal((n, r))
        X[:] = 0.0
        reqs.append(Request(int(k), A, B, X, arena))
    return reqs


def backward_error(req: Request) -> float:
    """max over RHS of ||b - A x||_1 / (||A||_1 ||x||_1 + ||b||_1) (MAGMA testers' normwise form)."""
    A, B, X = req.A, req.B, req.X
    if req.kind == SOLVE_CHOLESKY:
        A = np.tril(A) + np.tril(A, -1).T
    R = B - A @ X
    an = np.abs(A).sum(axis=0).max()
    num = np.abs(R).sum(axis=0)
    den = an * np.abs(X).sum(axis=0) + np.abs(B).sum(axis=0)
    return float((num / den).max())


def run_load(server: Server, reqs: list[Request], rate: float, seed: int = 0) -> dict:
    """Submits `reqs` at Poisson arrival times of the given rate (requests/s), waits for
    all, and returns throughput and latency percentiles."""
    rng = np.random.default_rng(seed + 17)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    arr_ns = (arrivals * 1e9).astype(np.int64)
    t0 = time.monotonic_ns() + 2_000_000
    sched = t0 + arr_ns
    done = {}
    lag = 0
    for i, r in enumerate(reqs):
        while time.monotonic_ns() < sched[i]:
            pass
        server.submit(r.kind, r.A, r.B, r.X, i)
        lag = max(lag, time.monotonic_ns() - int(sched[i]))
        if (i & 63) == 63:
            for tag, inf, _, td in zip(*server.poll()):
                done[int(tag)] = (int(inf), int(td))
    server.drain()
    while True:
        got = server.poll()
        if not len(got[0]):
            break
        for tag, inf, _, td in zip(*got):
            done[int(tag)] = (int(inf), int(td))
    assert len(done) == len(reqs), (len(done), len(reqs))
    t_done = np.array([done[i][1] for i in range(len(reqs))], np.int64)
    infos = np.array([done[i][0] for i in range(len(reqs))], np.int32)
    lat = (t_done - sched) / 1e6
    span = (t_done.max() - sched[0]) / 1e9
    return {
        "offered_rate": rate,
        "requests": len(reqs),
        "throughput": len(reqs) / span,
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()),
        "infos_nonzero": int((infos != 0).sum()),
        "max_submit_lag_ms": lag / 1e6,
        **server.stats(),
    }


def solve_alone(server: Server, req: Request) -> np.ndarray:
    """Runs one request with nothing else in flight and returns a copy of its result."""
    server.submit(req.kind, req.A, req.B, req.X, 0)
    server.drain()
    server.poll()
    return req.X.copy()


__all__ = ["Server", "Request", "make_requests", "run_load", "solve_alone", "backward_error",
           "SOLVE_LU", "SOLVE_CHOLESKY"]
