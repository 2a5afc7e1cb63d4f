"""The multi-GPU form of the benchmark is N independent replicas (the batched path has no
exchange step): each rank times its own batch, the job's time is the slowest rank's, and
rank 0 alone reports. This file covers that host logic with world size 2 over gloo, on CPU."""
import datetime
import os
import socket
import types


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        # rank r's own timings: step ms, e2e ms, the second arm's ms, and its accuracy-bar
        # miss flag (rank 1 missed): every rank must learn of a miss on any rank
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.0, float(rank == 1)], dist)
        dist.barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world2_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == {0: [2.0, 10.0, 0.0, 1.0], 1: [2.0, 10.0, 0.0, 1.0]}


def test_max_over_ranks_single_rank():
    import bench

    assert bench.max_over_ranks([3, 4.5, 0], None) == [3.0, 4.5, 0.0]


def test_reference_arm_other_ranks_do_no_work(capsys):
    import bench

    args = types.SimpleNamespace(workload="c3", steps=1, warmup=3)
    assert bench.run_reference(args, 1) is None
    assert capsys.readouterr().out == ""


def test_dist_setup_reference_arm_needs_no_process_group(monkeypatch):
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    rank, world, local, dist = bench.dist_setup(types.SimpleNamespace(impl="reference"))
    assert (rank, world, local, dist) == (1, 2, 1, None)


def test_accuracy_gate():
    """The metric's bar: every instance at backward error <= 1e-14 with info 0; a NaN
    backward error is a miss."""
    import torch

    import bench

    be = torch.tensor([1e-16, 9.9e-15, 2e-15], dtype=torch.float64)
    info = torch.zeros(3, dtype=torch.int32)
    g, ok = bench.accuracy_gate("x", be, info)
    assert ok and g == {"x_bwd_err_max": 9.9e-15, "x_over_bar": 0, "x_info_nonzero": 0}
    _, ok = bench.accuracy_gate("x", torch.tensor([1e-16, 1.1e-14], dtype=torch.float64), info[:2])
    assert not ok
    _, ok = bench.accuracy_gate("x", torch.tensor([1e-16, float("nan")], dtype=torch.float64), info[:2])
    assert not ok
    _, ok = bench.accuracy_gate("x", be, torch.tensor([0, 3, 0], dtype=torch.int32))
    assert not ok
