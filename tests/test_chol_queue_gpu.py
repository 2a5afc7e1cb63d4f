"""GPU parity tests of the one-launch variable-size Cholesky (the persistent queue kernel).

With the tuning switch on (the default), magma_d{potrf,potrs,posv}_vbatched run every
instance of order <= 512 from one device queue in a single launch; with it off, one
launch per size bucket. Both must give the oracle's bits: factors, solutions and info,
for lower and upper storage, one and several right-hand sides, non-positive-definite
instances in every size class, and batches whose instances all sit in one class (the
blocks never split, or split at once down to single warps)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from magma_b200 import _lib
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
N_VALUES = 21
QUEUE = 19   # index of the queue switch in the tuning table


def _set_queue(v):
    lib = _lib.load()
    vals = (C.c_int * N_VALUES)()
    assert lib.magma_b200_tuning_get(vals, N_VALUES) == N_VALUES
    old = vals[QUEUE]
    vals[QUEUE] = v
    assert lib.magma_b200_tuning_set(vals, N_VALUES) == 0
    return old


@pytest.fixture
def queue_switch():
    old = _set_queue(1)
    yield _set_queue
    _set_queue(old)


def _power_law_sizes(count, lo, hi, seed):
    u = T.uniform01(seed, 11, count)
    a, b = lo ** -0.5, hi ** -0.5
    return np.clip(np.round((a - u * (a - b)) ** -2), lo, hi).astype(np.int32)


def _problem(ns, nrhs, seed, bad=()):
    lda = ((ns + 3) // 4) * 4 + 1
    As = [np.zeros((max(n, 1), ld)) for n, ld in zip(ns, lda)]
    for i, n in enumerate(ns):
        if n:
            As[i][:n, :n] = T.spd_gram(int(n), seed, i)
    for i, k in bad:   # make leading minor k+1 of instance i non-positive
        As[i][k, k] = -1.0
    Bs = [T.normal(seed, 7000 + i, int(max(n, 1) * r)).reshape(r, max(n, 1)) for i, (n, r) in enumerate(zip(ns, nrhs))]
    ldb = np.array([max(n, 1) for n in ns], np.int32)
    return As, Bs, lda.astype(np.int32), ldb


def _run(cuda, As, Bs, ns, nrhs, lda, ldb, upper, factor, solve, fixed_max=True):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    gA, gB = VarBatch([a.copy() for a in As], cuda), VarBatch([b.copy() for b in Bs], cuda)
    mx = (int(ns.max()), int(nrhs.max())) if fixed_max else None
    info = mb.dposv_vbatched(gA, gB if solve else None, ns, nrhs if solve else None, lda, ldb if solve else None,
                             upper=upper, factor=factor, solve=solve, max_sizes=mx)
    info = info.cpu().numpy() if info is not None else None
    return info, gA.unpack(), gB.unpack()


def _oracle(As, Bs, ns, nrhs, lda, ldb, upper, solve):
    OA = [a.copy() for a in As]
    OB = [b.copy() for b in Bs]
    oinf = oracle.dposv_vbatched(OA, OB, ns, nrhs, lda, ldb, solve=solve, upper=upper)
    return oinf, OA, OB


def _tri(a, n, upper):
    return np.triu(a[:n, :n].T) if upper else np.tril(a[:n, :n].T)


def _compare(got, want, ns, factor, solve, upper):
    """Bit-identical factors, solutions and info. Where the factorisation stops (info = g + 1),
    LAPACK defines only info and the finished columns 0..g-1 of L: the blocked kernels, like
    LAPACK's blocked dpotrf, leave the columns past the failing panel without that panel's
    updates, so only those columns are compared and the solution is not."""
    ginf, GA, GB = got
    oinf, OA, OB = want
    if factor:
        assert np.array_equal(ginf, oinf)
    for i, n in enumerate(ns):
        failed = factor and oinf[i] > 0
        if factor:
            g, o = _tri(GA[i], n, upper), _tri(OA[i], n, upper)
            if failed:
                done = oinf[i] - 1
                g, o = (g.T, o.T) if upper else (g, o)
                g, o = g[:, :done], o[:, :done]
            assert np.array_equal(g, o), (i, n)
        if solve and not failed:
            assert np.array_equal(GB[i], OB[i]), (i, n)


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("mode", ["posv", "potrf", "potrs"])
def test_queue_matches_oracle_and_buckets(cuda, queue_switch, upper, mode):
    batch = 600
    ns = _power_law_sizes(batch, 1, 512, seed=21)
    ns[:8] = [512, 257, 256, 129, 128, 65, 64, 33]   # every class edge
    ns[8] = 0                                          # an empty instance
    nrhs = (1 + np.floor(T.uniform01(21, 12, batch) * 8)).astype(np.int32)
    factor, solve = mode != "potrs", mode != "potrf"
    bad = [(0, 300), (3, 100), (5, 40), (7, 20), (20, 0)] if factor else []
    assert all(k < ns[i] for i, k in bad)
    As, Bs, lda, ldb = _problem(ns, nrhs, 31, bad)
    want = _oracle(As, Bs, ns, nrhs, lda, ldb, upper, solve)
    if not factor:   # potrs starts from the oracle's factor and must reach the oracle's posv solution
        As = want[1]
    got_q = _run(cuda, As, Bs, ns, nrhs, lda, ldb, upper, factor, solve)
    _compare(got_q, want, ns, factor, solve, upper)
    queue_switch(0)
    got_b = _run(cuda, As, Bs, ns, nrhs, lda, ldb, upper, factor, solve)
    _compare(got_b, want, ns, factor, solve, upper)


@pytest.mark.parametrize("sizes", ["all512", "all4", "one_rhs", "with1024"])
def test_queue_edge_batches(cuda, queue_switch, sizes):
    if sizes == "all512":
        ns = np.full(40, 512, np.int32)
    elif sizes == "all4":
        ns = np.full(3000, 4, np.int32)
    elif sizes == "with1024":   # the 1024-thread bucket runs beside the queue
        ns = _power_law_sizes(300, 1, 512, seed=23)
        ns[[0, 50, 99]] = [1024, 700, 513]
    else:
        ns = _power_law_sizes(500, 1, 512, seed=24)
    nrhs = np.ones(len(ns), np.int32) if sizes == "one_rhs" else \
        (1 + np.floor(T.uniform01(25, 12, len(ns)) * 8)).astype(np.int32)
    As, Bs, lda, ldb = _problem(ns, nrhs, 33)
    want = _oracle(As, Bs, ns, nrhs, lda, ldb, False, True)
    got = _run(cuda, As, Bs, ns, nrhs, lda, ldb, False, True, True, fixed_max=(sizes != "all4"))
    _compare(got, want, ns, True, True, False)
