"""GPU parity tests of the variable-size batched LU (getrf / getrs / gesv _vbatched)
through the C ABI: factors, pivots, info and solutions bit-identical to the
oracle's dgetf2/dgetrs restatement instance by instance, for sizes across every
size bucket (register-resident and blocked kernels) in one call."""
import numpy as np
import pytest

import oracle
from magma_b200 import testing as T

pytestmark = pytest.mark.gpu


def _sizes(count, seed, nmax=700):
    u = T.uniform01(seed, 21, count)
    a, b = 1.0, nmax ** -0.5
    return np.clip(np.round((a - u * (a - b)) ** -2), 1, nmax).astype(np.int32)


@pytest.mark.parametrize("checked", [True, False])
def test_gesv_vbatched_bit_identical(cuda, checked):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    count = 300
    ns = _sizes(count, 3)
    ns[:3] = [1, 1024, 64]
    nrhs = (1 + np.floor(T.uniform01(3, 22, count) * 6)).astype(np.int32)
    lda = T.roundup(ns, 4).astype(np.int32)
    As = [np.zeros((n, l)) for n, l in zip(ns, lda)]
    Bs = [np.zeros((r, n)) for r, n in zip(nrhs, ns)]
    for i, n in enumerate(ns):
        As[i][:, :n] = T.uniform11(50 + i, 0, n * n).reshape(n, n)
        Bs[i][:, :] = T.uniform11(50 + i, 1, n * nrhs[i]).reshape(nrhs[i], n)
    As[5][:, :] = 0.0                                   # singular: info 1
    gA, gB = VarBatch(As, cuda), VarBatch(Bs, cuda)
    mx = None if checked else (int(ns.max()), int(nrhs.max()))
    ipiv, info = mb.dgesv_vbatched(gA, gB, ns, nrhs, lda, ns, max_sizes=mx)
    RA, RB = gA.unpack(), gB.unpack()
    ip, inf = ipiv.cpu().numpy(), info.cpu().numpy()
    for i, n in enumerate(ns):
        OA = As[i][None].copy()
        OB = Bs[i][None].copy()
        oip, oinf = oracle.dgesv_batched(OA, OB)
        assert inf[i] == oinf[0], i
        assert np.array_equal(ip[i, :n], oip[0]), i
        assert np.array_equal(RA[i], OA[0]), i
        if oinf[0] == 0:
            assert np.array_equal(RB[i], OB[0]), i
    assert inf[5] == 1


def test_getrf_getrs_vbatched_rectangular_and_trans(cuda):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    count = 120
    ms = _sizes(count, 7, 300)
    ns = _sizes(count, 8, 300)
    As = [T.uniform11(90 + i, 0, int(m * n)).reshape(n, m) for i, (m, n) in enumerate(zip(ms, ns))]
    gA = VarBatch(As, cuda)
    ipiv, info = mb.dgesv_vbatched(gA, None, ns, lda=ms, m=ms, solve=False)
    RA = gA.unpack()
    ip = ipiv.cpu().numpy()
    for i, (m, n) in enumerate(zip(ms, ns)):
        O = As[i][None].copy()
        oip, oinf = oracle.dgetrf_batched(O, int(m))
        k = min(m, n)
        assert np.array_equal(RA[i], O[0]), i
        assert np.array_equal(ip[i, :k], oip[0, :k]), i
        assert info[i].item() == oinf[0]
    # square instances: getrs NoTrans (bit-identical) and Trans (tolerance) on the factors
    sq = [i for i in range(count) if ms[i] == ns[i]] or [0]
    sqA = [As[i][:, :ns[i]].copy() if ms[i] == ns[i] else np.eye(3) for i in range(count)]
    n2 = np.array([ns[i] if ms[i] == ns[i] else 3 for i in range(count)], np.int32)
    F = [a[None].copy() for a in sqA]
    fp = []
    for f, n in zip(F, n2):
        p, _ = oracle.dgetrf_batched(f, int(n))
        fp.append(p[0])
    import torch
    P = torch.zeros((count, int(n2.max())), dtype=torch.int32)
    for i, p in enumerate(fp):
        P[i, :len(p)] = torch.from_numpy(p)
    P = P.to(cuda)
    for trans in (False, True):
        Bs = [T.uniform11(300 + i, 1, int(2 * n)).reshape(2, n) for i, n in enumerate(n2)]
        gF, gB = VarBatch([f[0] for f in F], cuda), VarBatch(Bs, cuda)
        mb.dgesv_vbatched(gF, gB, n2, [2] * count, n2, n2, factor=False, trans=trans, ipiv=P)
        RB = gB.unpack()
        for i, n in enumerate(n2):
            OB = Bs[i][None].copy()
            oracle.dgetrs_batched(F[i].copy(), fp[i][None].copy(), OB, trans=trans)
            if not trans:
                assert np.array_equal(RB[i], OB[0]), i
            else:
                assert np.abs(RB[i] - OB[0]).max() <= 64 * n * 2.3e-16 * max(np.abs(OB).max(), 1.0), i
    del sq


def test_getrf_vbatched_argument_errors(cuda):
    import magma_b200 as mb
    from magma_b200.api import VarBatch
    gA = VarBatch([np.eye(4), np.eye(3)], cuda)
    with pytest.raises(ValueError, match="-1"):
        mb.dgesv_vbatched(gA, None, [4, 3], lda=[4, 3], m=[4, -3], solve=False)
    with pytest.raises(ValueError, match="-4"):
        mb.dgesv_vbatched(gA, None, [4, 3], lda=[4, 2], solve=False)
