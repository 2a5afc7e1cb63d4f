"""GPU tests of the request loop (include/magma_b200_serve.h).

Continuous batching must not change any result: every request's solution is
BIT-IDENTICAL whether it ran alone or inside a micro-batch with other sizes and
kinds, because each instance runs the same size-bucket kernel in both cases.
Every solution meets the backward-error bar 1e-14, and admission keeps device
use within the memory budget.
"""
import numpy as np
import pytest

from magma_b200 import serve

pytestmark = pytest.mark.gpu


def _mix_then_alone(reqs, budget, streams, max_batch, rate):
    with serve.Server(budget, streams=streams, max_batch=max_batch) as sv:
        res = serve.run_load(sv, reqs, rate=rate, seed=1)
        mixed = [r.X.copy() for r in reqs]
    with serve.Server(budget, streams=1, max_batch=1) as sv:
        alone = []
        for r in reqs:
            r.X[:] = np.nan
            alone.append(serve.solve_alone(sv, r))
    return res, mixed, alone


def test_alone_equals_in_mix(cuda):
    reqs = serve.make_requests(64, seed=11)
    res, mixed, alone = _mix_then_alone(reqs, budget=1 << 30, streams=3, max_batch=64, rate=1e6)
    assert res["completed"] == len(reqs) and res["infos_nonzero"] == 0
    assert res["batches"] < len(reqs)            # requests were batched together
    for i, r in enumerate(reqs):
        assert np.array_equal(mixed[i], alone[i]), (i, r.kind, r.A.shape, r.B.shape)
        assert serve.backward_error(r) <= 1e-14, (i, r.kind, r.A.shape)


def test_admission_respects_budget(cuda):
    reqs = serve.make_requests(40, seed=12, n_lo=200, n_hi=600)
    need = max(8 * r.A.size + 8 * r.B.size + 4 * r.A.shape[0] + 3 * 256 for r in reqs)
    budget = 2 * need + (1 << 20)                # room for about two requests at a time
    res, mixed, alone = _mix_then_alone(reqs, budget=budget, streams=4, max_batch=32, rate=1e6)
    assert res["completed"] == len(reqs)
    assert 0 < res["peak_bytes"] <= budget
    for i, r in enumerate(reqs):
        assert np.array_equal(mixed[i], alone[i]), i
        assert serve.backward_error(r) <= 1e-14, i


def test_singular_request_reports_info(cuda):
    reqs = serve.make_requests(6, seed=13, n_lo=20, n_hi=90, lu_share=1.0)
    reqs[2].A[:, 5] = 0.0                         # zero column 6 -> info 6
    with serve.Server(1 << 28) as sv:
        for i, r in enumerate(reqs):
            sv.submit(r.kind, r.A, r.B, r.X, i)
        sv.drain()
        tags, infos, ts, td = sv.poll()
    got = dict(zip(tags.tolist(), infos.tolist()))
    assert got == {0: 0, 1: 0, 2: 6, 3: 0, 4: 0, 5: 0}
    assert (td >= ts).all()


def test_oversized_request_rejected(cuda):
    reqs = serve.make_requests(1, seed=14, n_lo=500, n_hi=500)
    with serve.Server(1 << 20) as sv:             # 1 MiB arena < one 500x500 matrix
        with pytest.raises(ValueError, match="-103"):
            sv.submit(reqs[0].kind, reqs[0].A, reqs[0].B, reqs[0].X, 0)
