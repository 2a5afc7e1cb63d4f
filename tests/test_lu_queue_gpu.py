"""GPU parity tests of the one-launch variable-size LU (the persistent queue kernel).

With the tuning switch on (it is off by default: the per-bucket launches measured
faster on the size mix tried), magma_dgetrf_vbatched and magma_dgesv_vbatched
run every instance with max(m, n) <= 512 from one device queue in a single launch; with
it off, one launch per size bucket. Both must give the oracle's bits: factors, pivots,
info and NoTrans solutions, for square and rectangular instances in every size class,
singular instances, one and several right-hand sides, and batches whose instances all sit
in one class."""
import ctypes as C

import numpy as np
import pytest

import oracle
from magma_b200 import _lib
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu
N_VALUES = 21
LU_QUEUE = 20   # index of the switch in the tuning table


def _set_switch(v):
    lib = _lib.load()
    vals = (C.c_int * N_VALUES)()
    assert lib.magma_b200_tuning_get(vals, N_VALUES) == N_VALUES
    old = vals[LU_QUEUE]
    vals[LU_QUEUE] = v
    assert lib.magma_b200_tuning_set(vals, N_VALUES) == 0
    return old


@pytest.fixture
def lu_switch():
    old = _set_switch(1)
    yield _set_switch
    _set_switch(old)


def _sizes(count, seed, nmax):
    u = T.uniform01(seed, 21, count)
    a, b = 1.0, nmax ** -0.5
    return np.clip(np.round((a - u * (a - b)) ** -2), 1, nmax).astype(np.int32)


def _gesv_case(cuda, ns, nrhs, seed, singular=(), fixed_max=True):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    lda = T.roundup(ns, 4).astype(np.int32) + 1
    As = [np.zeros((n, l)) for n, l in zip(ns, lda)]
    Bs = [np.zeros((r, n)) for r, n in zip(nrhs, ns)]
    for i, n in enumerate(ns):
        As[i][:, :n] = T.uniform11(seed + i, 0, n * n).reshape(n, n)
        Bs[i][:, :] = T.uniform11(seed + i, 1, n * nrhs[i]).reshape(nrhs[i], n)
    for i in singular:
        As[i][:, :] = 0.0
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    mx = (int(ns.max()), int(nrhs.max())) if fixed_max else None
    ipiv, info = mb.dgesv_vbatched(gA, gB, ns, nrhs, lda, ns, max_sizes=mx)
    RA, RB = gA.unpack(), gB.unpack()
    ip, inf = ipiv.cpu().numpy(), info.cpu().numpy()
    for i, n in enumerate(ns):
        OA = As[i][None].copy()
        OB = Bs[i][None].copy()
        oip, oinf = oracle.dgesv_batched(OA, OB)
        assert inf[i] == oinf[0], i
        assert np.array_equal(ip[i, :n], oip[0]), i
        assert np.array_equal(RA[i], OA[0]), i   # the padding rows past n untouched too
        if oinf[0] == 0:
            assert np.array_equal(RB[i], OB[0]), i
    return inf


def test_lu_queue_gesv_matches_oracle_and_buckets(cuda, lu_switch):
    count = 400
    ns = _sizes(count, 5, 512)
    ns[:8] = [512, 257, 256, 129, 128, 65, 64, 33]     # every class edge
    nrhs = (1 + np.floor(T.uniform01(5, 22, count) * 8)).astype(np.int32)
    inf = _gesv_case(cuda, ns, nrhs, 300, singular=(1, 4, 6, 9))
    assert inf[1] == 1 and inf[4] == 1 and inf[6] == 1
    lu_switch(0)
    _gesv_case(cuda, ns, nrhs, 300, singular=(1, 4, 6, 9))


@pytest.mark.parametrize("sizes", ["all512", "all5", "one_rhs", "with1024"])
def test_lu_queue_gesv_edge_batches(cuda, lu_switch, sizes):
    if sizes == "all512":
        ns = np.full(30, 512, np.int32)
    elif sizes == "all5":
        ns = np.full(2000, 5, np.int32)
    elif sizes == "with1024":   # the 1024-thread bucket runs beside the queue
        ns = _sizes(200, 6, 512)
        ns[[0, 40, 77]] = [1024, 700, 513]
    else:
        ns = _sizes(300, 7, 512)
    nrhs = np.ones(len(ns), np.int32) if sizes == "one_rhs" else \
        (1 + np.floor(T.uniform01(8, 22, len(ns)) * 4)).astype(np.int32)
    _gesv_case(cuda, ns, nrhs, 700, fixed_max=(sizes != "all5"))


def test_lu_queue_getrf_rectangular(cuda, lu_switch):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    count = 160
    ms = _sizes(count, 9, 512)
    ns = _sizes(count, 10, 512)
    ms[:4], ns[:4] = [512, 20, 300, 64], [40, 512, 64, 300]
    As = [T.uniform11(900 + i, 0, int(m * n)).reshape(n, m) for i, (m, n) in enumerate(zip(ms, ns))]
    for flag in (1, 0):
        lu_switch(flag)
        gA = VarBatch(As, cuda)
        ipiv, info = mb.dgesv_vbatched(gA, None, ns, lda=ms, m=ms, solve=False)
        RA = gA.unpack()
        ip, inf = ipiv.cpu().numpy(), info.cpu().numpy()
        for i, (m, n) in enumerate(zip(ms, ns)):
            O = As[i][None].copy()
            oip, oinf = oracle.dgetrf_batched(O, int(m))
            k = min(m, n)
            assert np.array_equal(RA[i], O[0]), (flag, i)
            assert np.array_equal(ip[i, :k], oip[0, :k]), (flag, i)
            assert inf[i] == oinf[0], (flag, i)
