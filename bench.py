#!/usr/bin/env python
"""Benchmark of the batched dense solvers (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch of synthetic input:
  c1   plain FP64 LU + solve: magma_dgesv_batched on 10,000 x (32x32), 1 RHS,
       entries U[-1,1] (seeded).

Timing: W untimed steps, then exactly K steps between a barrier +
cudaDeviceSynchronize on both sides, measured with CUDA events on the
library's stream, max over ranks. Each step factors a different input buffer
from a ring whose total size exceeds the 126 MB L2, so a step never finds its
inputs in L2. N > 1 runs one replica per GPU on its own batch (independent
instances, no collective on the data path; scaling "weak").

`value` has the inputs resident in HBM; `e2e` is the same metric through the
public C ABI with the inputs copied from pinned host memory and the results
(x, ipiv, info) copied back inside every timed step. `cpu_baseline` times the
reference's own CPU path (an OpenMP loop of LAPACK dgesv, one instance per
iteration, testing_zgetrf_batched.cpp:188-206) on this host's cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/s at bwd err ≤1e-14: mixed-prec vs FP64 on 1 B200; p50/p99 latency"
L2_BYTES = 126 * 2**20


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "src": "fallback"}


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/ (None if absent)."""
    f = ROOT / "profiles" / f"{kernel}__{workload}.md"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch\s*=\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.index = gpu_id
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.15)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        self.proc.wait()
        self.out.flush()
        rows = [r.split(",") for r in Path(self.out.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 4 + k and r[4 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------ workloads
class C1DgesvSmall:
    """Plain FP64 LU + solve, 10,000 x (32x32), 1 RHS (magma_dgesv_batched)."""
    name = "c1_dgesv_batched_32x32"
    kernel = "gesv_small_kernel"
    dtype = "f64"

    def __init__(self, dev, batch=10000, n=32, nrhs=1, seed=1):
        import numpy as np
        import torch

        from magma_b200 import testing as T

        self.np, self.torch = np, torch
        self.dev, self.batch, self.n, self.nrhs = dev, batch, n, nrhs
        self.A_np, self.B_np = T.lu_uniform(batch, n, nrhs, seed=seed)
        step_bytes = 8 * batch * (n * n + n * nrhs)
        self.ring = max(2, -(-3 * L2_BYTES // step_bytes))     # ring larger than L2 (x3)
        self.A = [torch.from_numpy(self.A_np).to(dev) for _ in range(self.ring)]
        self.B = [torch.from_numpy(self.B_np).to(dev) for _ in range(self.ring)]
        self.ipiv = torch.zeros((batch, n), dtype=torch.int32, device=dev)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        from magma_b200.api import ptr_array

        self.pA = [ptr_array(a) for a in self.A]
        self.pB = [ptr_array(b) for b in self.B]
        self.pP = ptr_array(self.ipiv)

    # algorithmic counts (MAGMA testing/flops.h FLOPS_DGETRF + FLOPS_DGETRS; bytes read/written once)
    def units(self):
        return self.batch

    def bytes_per_unit(self):
        n, r = self.n, self.nrhs
        return 2 * 8 * n * n + 2 * 8 * n * r + 4 * n + 4

    def launches_per_step(self):
        return 1

    def step(self, q, i):
        k = i % self.ring
        return q.lib.magma_dgesv_batched(self.n, self.nrhs, C.c_void_p(self.pA[k].data_ptr()), self.n,
                                         C.c_void_p(self.pP.data_ptr()), C.c_void_p(self.pB[k].data_ptr()),
                                         self.n, C.c_void_p(self.info.data_ptr()), self.batch, q.handle)

    def validate(self, q):
        """Fresh solve of the pristine batch; returns the max normwise backward error (checked on host)."""
        from magma_b200 import testing as T

        A = self.torch.from_numpy(self.A_np).to(self.dev)
        B = self.torch.from_numpy(self.B_np).to(self.dev)
        from magma_b200.api import dgesv_batched

        dgesv_batched(A, B, queue=q)
        q.sync()
        return float(T.backward_error(self.A_np, B.cpu().numpy(), self.B_np, self.n).max())

    # end-to-end through the C ABI with host buffers
    def e2e_setup(self):
        t = self.torch
        self.hA = t.from_numpy(self.A_np).pin_memory()
        self.hB = t.from_numpy(self.B_np).pin_memory()
        self.hX = t.empty_like(self.hB).pin_memory()
        self.hP = t.empty((self.batch, self.n), dtype=t.int32).pin_memory()
        self.hI = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.h2d = self.hA.numel() * 8 + self.hB.numel() * 8
        self.d2h = self.hX.numel() * 8 + self.hP.numel() * 4 + self.hI.numel() * 4

    def e2e_step(self, q, i):
        k = i % self.ring
        self.A[k].copy_(self.hA, non_blocking=True)
        self.B[k].copy_(self.hB, non_blocking=True)
        self.step(q, i)
        self.hX.copy_(self.B[k], non_blocking=True)
        self.hP.copy_(self.ipiv, non_blocking=True)
        self.hI.copy_(self.info, non_blocking=True)

    # reference CPU path on a bounded sample
    def cpu_reference(self, seconds=10.0, nthreads=None):
        import oracle

        sample = min(self.batch, 10000)
        A0, B0 = self.A_np[:sample], self.B_np[:sample]
        done, t_total = 0, 0.0
        while t_total < seconds:
            A, B = A0.copy(), B0.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgesv_batched(A, B, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += sample
        return done / t_total, done, (nthreads or oracle.max_threads())


WORKLOADS = {"c1": C1DgesvSmall}


# ---------------------------------------------------------------------- main
def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if args.impl == "reference":
            return rank, world, local, None
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        return rank, world, local, dist
    return rank, world, local, None


def run_reference(args, rank, world):
    """The reference's CPU implementation (LAPACK loop) on this host; rank 0 only."""
    if rank != 0:
        return
    import numpy as np  # noqa: F401

    import oracle

    W = WORKLOADS[args.workload]
    from magma_b200 import testing as T

    nthreads = oracle.max_threads()
    if args.workload == "c1":
        sample = 10000
        A0, B0 = T.lu_uniform(sample, 32, 1, seed=1)
        for _ in range(args.warmup):
            oracle.lapack_dgesv_batched(A0.copy(), B0.copy(), nthreads=nthreads)
        times = []
        for _ in range(args.steps):
            A, B = A0.copy(), B0.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgesv_batched(A, B, nthreads=nthreads)
            times.append(time.perf_counter() - t0)
        total = sum(times)
        value = sample * args.steps / total
        ms = 1e3 * total / args.steps
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": W.dtype, "data": "synthetic (seeded U[-1,1])",
        "config": {"workload": W.name, "batch": sample, "n": 32, "nrhs": 1},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{sample} instances per step; LAPACK dgesv (OpenBLAS 0.3.30, scipy) in an "
                                   f"OpenMP loop, 1 BLAS thread per instance"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c1")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    defaults = {"c1": (20000, 50)}
    if args.steps is None:
        args.steps = defaults[args.workload][0] if args.impl == "ours" else 20
    if args.warmup is None:
        args.warmup = defaults[args.workload][1] if args.impl == "ours" else 3
    args.warmup = max(args.warmup, 3)

    rank, world, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    import magma_b200 as mb
    from magma_b200.api import Queue

    mb.load()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    W = WORKLOADS[args.workload](dev)
    with torch.cuda.stream(stream):
        q = Queue(stream, local)
        bwd = W.validate(q)
        for i in range(args.warmup):
            W.step(q, i)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        # nvidia-smi ignores CUDA_VISIBLE_DEVICES: address the GPU by its UUID
        clocks = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(dev).uuid))
        clocks.start()
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            rc = W.step(q, i)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        clk = clocks.stop()
        assert rc == 0, f"library returned {rc}"
        ms_total = e0.elapsed_time(e1)
        # end to end (host buffers, copies inside each step)
        W.e2e_setup()
        ke = max(3, min(args.steps, 200))
        for i in range(3):
            W.e2e_step(q, i)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for i in range(ke):
            W.e2e_step(q, i)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        ms_e2e = f0.elapsed_time(f1)
    if dist:
        t = torch.tensor([ms_total, ms_e2e, bwd], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total, ms_e2e, bwd = (float(v) for v in t.tolist())
    units = W.units() * world
    value = units * args.steps / (ms_total * 1e-3)
    e2e_value = units * ke / (ms_e2e * 1e-3)
    if rank == 0:
        peaks = measured_peaks()
        per_launch_ms = ms_total / (args.steps * W.launches_per_step())
        alg_bytes = W.bytes_per_unit() * W.units()
        achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
        traffic = profile_traffic(W.kernel, W.name)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": W.dtype,
            "data": "synthetic (seeded U[-1,1], splitmix64)",
            "config": {"workload": W.name, "batch_per_gpu": W.batch, "n": W.n, "nrhs": W.nrhs,
                       "parallelism": f"replicas x{world}",
                       "l2": f"ring of {W.ring} distinct input buffers ({W.ring} x "
                             f"{8 * W.batch * (W.n * W.n + W.n * W.nrhs) / 2**20:.0f} MiB) > L2"},
            "bwd_err_max": bwd,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "kernel": W.kernel, "peak_src": peaks["src"],
                         "alg_bytes_per_launch": alg_bytes},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": W.h2d,
                    "d2h_bytes_per_step": W.d2h, "steps": ke},
            "gpu_launches": args.steps * W.launches_per_step(),
            "clocks": clk,
        }
        if not args.no_cpu_baseline and world == 1:
            v, done, cores = W.cpu_reference()
            line["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                                    "sample": f"{done} solves (10,000-instance batches, same inputs); LAPACK dgesv "
                                              f"(OpenBLAS 0.3.30, scipy) in an OpenMP loop, 1 BLAS thread each"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
