#!/usr/bin/env python
"""Benchmark of the batched dense solvers (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch of synthetic input.
Workloads (the default is the one the metric is quoted on):
  c3  mixed-precision dgesv: 2,048 x (256x256), A = U diag(sigma) V^T with Haar U, V and
      log-uniform sigma (kappa log-uniform in [1e2, 1e6]), 4 RHS ~ N(0,1);
      magma_dsgesv_batched (FP32 LU + FP64 refinement + FP64 fallback) against the
      plain FP64 form magma_dgesv_batched on the same inputs.       [default]
  c1  plain FP64 LU + solve: magma_dgesv_batched on 10,000 x (32x32), 1 RHS, U[-1,1].
  c2  gemm_vbatched: 20,000 instances, M, N, K ~ U{8..128}, alpha 1, beta 0.5, FP64 with
      the FP32 arm beside (GFLOP/s).
  c4  posv_vbatched: 50,000 SPD instances, n power-law on [4, 512], 1-8 RHS, FP64 and
      FP32-factor + FP64-refinement (dsposv_vbatched), each replayed as one CUDA graph
      (solves/s).
  c5  the request loop: Poisson arrivals swept 1e3..1e5 req/s, 70% LU / 30% Cholesky,
      n log-uniform on [8, 1024], 1-16 RHS, 40 GB admission budget; throughput and
      p50/p99 latency at 1e4 req/s, the sweep beside.
  qr  Householder QR: magma_dgeqrf_batched on 10,000 x (64x64), U[-1,1] (factorizations/s).
  getri  LU + out-of-place inverse (getrf + getri_outofplace) on 10,000 x (32x32) (inverses/s).
  nopiv  gesv_nopiv_batched on 10,000 x (32x32) diagonally dominant, 1 RHS, with
      gesv_rbt_batched on the same inputs beside (solves/s).
  trsm  trsm_vbatched (left, lower, no-trans, non-unit) on 20,000 instances, M, N ~ U{8..128},
      with trmm_vbatched on the same operands beside (GFLOP/s).

Timing: W untimed steps, then exactly K steps between a barrier + device
synchronisation on both sides, measured with CUDA events on the library's
stream, max over ranks. The c3 inputs (1 GiB of A) exceed the 126 MB L2; c3
re-creates its overwritten inputs on the device between steps, outside the
per-step event brackets (the FP64 form overwrites A with its factors); c1
cycles through a ring of input buffers larger than L2 (each slot reset to the
original inputs after use, outside the brackets). Every workload whose metric is
"solves/s at bwd err <= 1e-14" checks the outputs of its last timed step (and of
its second arm's) against that bar on every instance, with info == 0; a miss
exits non-zero with no JSON line. N > 1 runs one replica
per GPU on its own batch (instances are independent; no collective on the
data path; scaling "weak").

`value` has the inputs resident in HBM; `e2e` is the same metric through the
public C ABI with the inputs copied from pinned host memory and the results
copied back inside every timed step. `cpu_baseline` (and `--impl reference`)
time the reference's own CPU path -- host LAPACK called per instance in an
OpenMP loop (testing/testing_zgetrf_batched.cpp:188-206) -- on this host.
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
# more hardware work queues than the driver's default 8 for the library's streams
# (set before torch creates the CUDA context; a value already set is kept)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "solves/s at bwd err ≤1e-14: mixed-prec vs FP64 on 1 B200; p50/p99 latency"
L2_BYTES = 126 * 2**20
FP64_NOMINAL_TFLOPS = 37.0   # B200 dense FP64 (CUDA cores / DMMA), nominal
BWD_BAR = 1e-14              # the metric's accuracy bar: normwise backward error per instance


def accuracy_gate(tag, be, info):
    """The metric's bar on one step's outputs: every instance's normwise backward error
    <= BWD_BAR and info == 0 (the inputs are well-posed). `be` and `info` are tensors over
    the instances. Returns ({tag_bwd_err_max, tag_info_nonzero, tag_ok}, ok)."""
    worst = float(be.max().item()) if be.numel() else 0.0
    bad_be = int((~(be <= BWD_BAR)).sum().item())          # NaN counts as a miss
    nz = int((info != 0).sum().item())
    ok = bad_be == 0 and nz == 0
    return {f"{tag}_bwd_err_max": worst, f"{tag}_over_bar": bad_be, f"{tag}_info_nonzero": nz}, ok


def host_cpu() -> dict:
    """The host's CPU model and logical CPU count (recorded beside every CPU baseline)."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


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
        self.gpu_id = gpu_id
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
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

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[0]) for r in rows) if v is not None]
        smax = [v for v in (num(r[1]) for r in rows if len(r) > 1) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 4 + k and r[4 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def timed(stream, fn, steps):
    """ms for `steps` calls of fn(i), CUDA events on `stream`."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        fn(i)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def timed_restore(stream, fn, restore, steps):
    """ms summed over `steps` calls of fn(i), each bracketed by its own CUDA events on
    `stream`; restore(i) re-creates the step's overwritten inputs between the brackets
    (on the device, outside the timed intervals)."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        restore(i)
        ev[i][0].record(stream)
        fn(i)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def vp(t):
    return C.c_void_p(t.data_ptr())


# ------------------------------------------------------------------ workloads
class C3Mixed:
    """Mixed-precision dgesv vs plain FP64 on 2,048 x (256x256), kappa in [1e2, 1e6], 4 RHS."""
    unit = "solves/s"
    dtype = "f32-factor+f64-refine"
    data = "synthetic: A = U diag(sigma) V^T, Haar U,V (QR of seeded Gaussians), log-uniform sigma, B ~ N(0,1)"

    def __init__(self, dev, batch=2048, n=256, nrhs=4, seed=3):
        import torch

        from magma_b200.api import ptr_array
        from magma_b200.testing import svd_logrand_torch

        self.torch, self.dev, self.batch, self.n, self.nrhs = torch, dev, batch, n, nrhs
        self.name = f"c3_dsgesv_batched_{batch}x{n}_kappa1e2-1e6_nrhs{nrhs}"
        self.A0, self.B0, self.kappa = svd_logrand_torch(batch, n, 1e2, 1e6, nrhs, seed, dev)
        self.A = self.A0.clone()
        self.B = self.B0.clone()
        self.X = torch.empty_like(self.B)
        self.ipiv = torch.zeros((batch, n), dtype=torch.int32, device=dev)
        self.iter = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.A64 = self.A0.clone()
        self.B64 = self.B0.clone()
        self.pA, self.pB, self.pX = ptr_array(self.A), ptr_array(self.B), ptr_array(self.X)
        self.pP = ptr_array(self.ipiv)
        self.pA64, self.pB64 = ptr_array(self.A64), ptr_array(self.B64)
        self.l2 = f"inputs {batch * n * n * 8 / 2**30:.2f} GiB > L2 (126 MB)"

    def units(self):
        return self.batch

    # algorithmic bytes per solve for the mixed path: read A and B, write X and ipiv
    def bytes_per_unit(self):
        n, r = self.n, self.nrhs
        return 8 * n * n + 2 * 8 * n * r + 4 * n

    def launches_per_step(self):
        return 4   # tensor-core LU + refinement (one kernel), fallback getrf, copy, fallback getrs

    def step(self, q, i):
        n = self.n
        return q.lib.magma_dsgesv_batched(n, self.nrhs, vp(self.pA), n, vp(self.pP), vp(self.pB), n, vp(self.pX), n,
                                          vp(self.iter), vp(self.info), self.batch, q.handle)

    def restore(self, i):
        self.A.copy_(self.A0)

    alt_name = "fp64"

    def config_extra(self):
        return {"n": self.n, "nrhs": self.nrhs}

    def ratios(self, value, alt_value):
        return {"mixed_over_fp64": value / alt_value}

    def restore_alt(self, i):
        self.A64.copy_(self.A0)
        self.B64.copy_(self.B0)

    def step_alt(self, q, i):
        n = self.n
        return q.lib.magma_dgesv_batched(n, self.nrhs, vp(self.pA64), n, vp(self.pP), vp(self.pB64), n,
                                         vp(self.info), self.batch, q.handle)

    def validate(self, q):
        from magma_b200.testing import backward_error_torch

        t = self.torch
        self.A.copy_(self.A0)
        rc = self.step(q, 0)
        q.sync()
        assert rc == 0, rc
        be_mixed = backward_error_torch(self.A0, self.X, self.B0).max().item()
        it = self.iter.cpu()
        hist = {int(k): int(v) for k, v in zip(*t.unique(it, return_counts=True))}
        A, B = self.A0.clone(), self.B0.clone()
        from magma_b200.api import dgesv_batched

        dgesv_batched(A, B, queue=q)
        q.sync()
        be_64 = backward_error_torch(self.A0, B, self.B0).max().item()
        self.A.copy_(self.A0)
        return {"bwd_err_max_mixed": be_mixed, "bwd_err_max_fp64": be_64, "iter_hist": hist}

    def check_last(self, q):
        """The bar on the last timed mixed step's outputs (X, info) for every instance."""
        from magma_b200.testing import backward_error_torch

        q.sync()
        return accuracy_gate("last_step_mixed", backward_error_torch(self.A0, self.X, self.B0).amax(dim=1),
                             self.info)

    def check_last_alt(self, q):
        """The bar on the last timed FP64 step's outputs (B overwritten by X, info)."""
        from magma_b200.testing import backward_error_torch

        q.sync()
        return accuracy_gate("last_step_fp64", backward_error_torch(self.A0, self.B64, self.B0).amax(dim=1),
                             self.info)

    def dominant_kernel(self, q, stream, reps=5):
        """Per-stage device times of the mixed step (queue stage timing: CUDA events the
        library records on its stream between the LU, refinement and fallback stages);
        the roofline is quoted for the dominant stage."""
        t = self.torch
        n, r, batch = self.n, self.nrhs, self.batch
        assert q.lib.magma_b200_stage_timing(q.handle, 1) == 0
        acc = [0.0, 0.0, 0.0]
        buf = (C.c_float * 8)()
        for i in range(reps):
            self.restore(i)
            self.step(q, i)
            k = q.lib.magma_b200_stage_times(q.handle, buf, 8)
            assert k == 3, k
            for j in range(3):
                acc[j] += buf[j] / reps
        q.lib.magma_b200_stage_timing(q.handle, 0)
        it = self.iter.cpu().clamp(min=0).to(t.float64)
        passes = float((it + 1).sum())
        lu_flops = batch * (2.0 / 3.0) * n ** 3
        refine_bytes = passes * 12.0 * n * n + batch * 16.0 * n * r
        stages = {"lu_ms": acc[0], "refine_ms": acc[1], "fallback_ms": acc[2]}
        if acc[1] < 0.05 * acc[0]:
            # one kernel factors on the tensor cores and refines in FP64: quoted against HBM
            # with the algorithm's compulsory bytes, A read by the factorisation and again by
            # every refinement pass ((1 + k) 8 n^2 bytes per solve after k passes), B read and X written
            stages = {"lu_and_refine_ms": acc[0], "fallback_ms": acc[2]}
            return {"kernel": "lu_tf32x3_kernel (tcgen05 split-TF32 LU + FP64 refinement, one block per instance)",
                    "ms": acc[0], "alg_bytes": (batch + passes) * 8.0 * n * n + batch * 16.0 * n * r,
                    "tflops": lu_flops / acc[0] / 1e9, "stages": stages,
                    "alg_note": "(1 + passes) 8 n^2 + 16 n nrhs B per instance, passes = iter + 1; the LU's 2/3 n^3 "
                                "flops on the tensor cores take under 1% of the kernel at the measured BF16 peak"}
        if acc[1] >= acc[0]:
            return {"kernel": "dsgesv_refine_kernel<256,4> (FP32 solves + FP64 residuals)", "ms": acc[1],
                    "alg_bytes": refine_bytes, "tflops": None, "stages": stages,
                    "alg_note": "12 n^2 B per refinement pass (A in FP64 + LU in FP32), passes = iter + 1"}
        return {"kernel": "lu_tf32x3_kernel (tcgen05 split-TF32 LU, TMEM-resident)", "ms": acc[0],
                "alg_flops": lu_flops, "tflops": lu_flops / acc[0] / 1e9, "stages": stages,
                "alg_bytes": batch * (8.0 * n * n + 4.0 * n * n + 4 * n)}

    def e2e_setup(self):
        t = self.torch
        self.hA = self.A0.cpu().pin_memory()
        self.hB = self.B0.cpu().pin_memory()
        self.hX = t.empty(self.B0.shape, dtype=t.float64).pin_memory()
        self.hI = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.hF = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.h2d = self.hA.numel() * 8 + self.hB.numel() * 8
        self.d2h = self.hX.numel() * 8 + 8 * self.batch

    e2e_api = "magma_b200_host_solve (C++; Python binding HostDsgesv), 8 chunks: uploads, solves and read-backs overlapped"

    def e2e_step(self, q, i):
        if getattr(self, "pipe", None) is None:
            from magma_b200.api import HostDsgesv

            self.pipe = HostDsgesv(self.batch, self.n, self.nrhs, chunks=8, queue=q)
        self.pipe(self.hA, self.hB, self.hX, self.hI, self.hF)

    def cpu_reference(self, seconds=10.0, nthreads=None, sample=512):
        """LAPACK dsgesv (the CPU mixed-precision solver) per instance, bounded sample."""
        import oracle

        A0 = self.A0[:sample].cpu().numpy().copy()
        B0 = self.B0[:sample].cpu().numpy().copy()
        done, t_total = 0, 0.0
        while t_total < seconds:
            A = A0.copy()
            t0 = time.perf_counter()
            X, ip, it, inf = oracle.lapack_dsgesv_batched(A, B0, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += sample
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} solves ({sample}-instance slices of the same inputs, re-run); LAPACK dsgesv " \
            f"(OpenBLAS 0.3.30, scipy) in an OpenMP loop, 1 BLAS thread each"


class C1DgesvSmall:
    """Plain FP64 LU + solve, 10,000 x (32x32), 1 RHS (magma_dgesv_batched)."""
    name = "c1_dgesv_batched_10000x32_nrhs1"
    unit = "solves/s"
    dtype = "f64"
    data = "synthetic: seeded U[-1,1] (splitmix64)"

    def __init__(self, dev, batch=10000, n=32, nrhs=1, seed=1):
        import torch

        from magma_b200 import testing as T
        from magma_b200.api import ptr_array

        self.torch, self.dev, self.batch, self.n, self.nrhs = torch, dev, batch, n, nrhs
        self.A_np, self.B_np = T.lu_uniform(batch, n, nrhs, seed=seed)
        step_bytes = 8 * batch * (n * n + n * nrhs)
        self.ring = max(2, -(-3 * L2_BYTES // step_bytes))
        self.A0 = torch.from_numpy(self.A_np).to(dev)
        self.B0 = torch.from_numpy(self.B_np).to(dev)
        self.A = [self.A0.clone() for _ in range(self.ring)]
        self.B = [self.B0.clone() for _ in range(self.ring)]
        self.ipiv = torch.zeros((batch, n), dtype=torch.int32, device=dev)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.pA = [ptr_array(a) for a in self.A]
        self.pB = [ptr_array(b) for b in self.B]
        self.pP = ptr_array(self.ipiv)
        self.l2 = (f"ring of {self.ring} distinct input buffers ({step_bytes / 2**20:.0f} MiB each) > L2, each reset "
                   f"to the original inputs after use, outside the per-step event brackets")

    def units(self):
        return self.batch

    def config_extra(self):
        return {"n": self.n, "nrhs": self.nrhs}

    def bytes_per_unit(self):
        n, r = self.n, self.nrhs
        return 2 * 8 * n * n + 2 * 8 * n * r + 4 * n + 4

    def launches_per_step(self):
        return 1

    def restore(self, i):
        """Step i reads ring slot i % ring. restore(0) resets every slot to the original
        inputs; restore(i) resets the slot step i-1 used, which is next read ring-1 steps
        later (more than twice L2 of traffic in between), so every step solves the original
        systems from HBM."""
        slots = range(self.ring) if i == 0 else [(i - 1) % self.ring]
        for k in slots:
            self.A[k].copy_(self.A0)
            self.B[k].copy_(self.B0)

    def step(self, q, i):
        k = i % self.ring
        self.last = k
        return q.lib.magma_dgesv_batched(self.n, self.nrhs, vp(self.pA[k]), self.n, vp(self.pP), vp(self.pB[k]),
                                         self.n, vp(self.info), self.batch, q.handle)

    def check_last(self, q):
        """The bar on the last timed step's outputs (its ring slot's X, info) for every instance."""
        from magma_b200.testing import backward_error_torch

        q.sync()
        return accuracy_gate("last_step_fp64", backward_error_torch(self.A0, self.B[self.last], self.B0).amax(dim=1),
                             self.info)

    def validate(self, q):
        from magma_b200 import testing as T
        from magma_b200.api import dgesv_batched

        A = self.torch.from_numpy(self.A_np).to(self.dev)
        B = self.torch.from_numpy(self.B_np).to(self.dev)
        dgesv_batched(A, B, queue=q)
        q.sync()
        return {"bwd_err_max_fp64": float(T.backward_error(self.A_np, B.cpu().numpy(), self.B_np, self.n).max())}

    def dominant_kernel(self, q, stream, reps=200):
        ms = timed(stream, lambda i: self.step(q, i), reps) / reps
        return {"kernel": "gesv_small_kernel<double,32,1,1>", "ms": ms, "alg_bytes": self.bytes_per_unit() * self.batch,
                "tflops": None}

    def extras(self, q, stream, reps=50):
        """The same steps replayed from one captured CUDA graph (one launch per ring buffer):
        launch overhead out of the picture."""
        t = self.torch
        try:
            g = t.cuda.CUDAGraph()
            with t.cuda.graph(g, stream=stream):
                for k in range(self.ring):
                    assert self.step(q, k) == 0
            g.replay()
            t.cuda.synchronize()
            ms = timed(stream, lambda i: g.replay(), reps) / (reps * self.ring)
            del g
        except Exception as e:   # reported, not fatal: the eager numbers stand on their own
            t.cuda.synchronize()
            return {"graph_replay": {"error": str(e)[:200]}}
        return {"graph_replay": {"ms_per_step": ms, "solves_per_s": self.batch / (ms * 1e-3),
                                 "steps_per_graph": self.ring}}

    def e2e_setup(self):
        t = self.torch
        self.hA = t.from_numpy(self.A_np).pin_memory()
        self.hB = t.from_numpy(self.B_np).pin_memory()
        self.hX = t.empty_like(self.hB).pin_memory()
        self.hP = t.empty((self.batch, self.n), dtype=t.int32).pin_memory()
        self.hI = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.h2d = self.hA.numel() * 8 + self.hB.numel() * 8
        self.d2h = self.hX.numel() * 8 + self.hP.numel() * 4 + self.hI.numel() * 4

    e2e_api = "magma_b200_host_solve (C++; Python binding HostDgesv), 4 chunks: uploads, solves and read-backs overlapped"

    def e2e_step(self, q, i):
        if getattr(self, "pipe", None) is None:
            from magma_b200.api import HostDgesv

            self.pipe = HostDgesv(self.batch, self.n, self.nrhs, chunks=4, queue=q)
        self.pipe(self.hA, self.hB, self.hX, self.hP, self.hI)

    def cpu_reference(self, seconds=10.0, nthreads=None):
        import oracle

        done, t_total = 0, 0.0
        while t_total < seconds:
            A, B = self.A_np.copy(), self.B_np.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgesv_batched(A, B, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += self.batch
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} solves (10,000-instance batches, same inputs); LAPACK dgesv (OpenBLAS 0.3.30, scipy) " \
            f"in an OpenMP loop, 1 BLAS thread each"



class C2GemmVbatched:
    """magmablas_dgemm_vbatched (and the sgemm arm) on 20,000 instances, M, N, K ~ U{8..128}."""
    unit = "GFLOP/s"
    dtype = "f64"
    metric = "gemm_vbatched GFLOP/s (FP64; FP32 arm beside)"
    data = "synthetic: M, N, K ~ U{8..128} (splitmix64), A, B, C ~ N(0,1) (torch seeded)"
    alt_name = "fp32"

    def __init__(self, dev, batch=20000, seed=2):
        import numpy as np
        import torch

        from magma_b200 import testing as T

        self.torch, self.dev, self.batch = torch, dev, batch
        self.name = f"c2_gemm_vbatched_{batch}_MNK8-128_alpha1_beta0.5"
        M, N, K = T.gemm_sizes(batch, 8, 128, seed=seed)
        r8 = lambda v: ((v + 7) // 8) * 8
        self.M, self.N, self.K = M, N, K
        self.lda, self.ldb, self.ldc = r8(M), r8(K), r8(M)
        self.flops = float((2.0 * M.astype(np.float64) * N * K).sum())
        self.bytes64 = float(8 * (M.astype(np.float64) * K + K * N + 2 * M * N).sum())
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        self.bufs = {}
        for dt, tag in ((torch.float64, "d"), (torch.float32, "s")):
            parts = {}
            for name, rows, cols in (("A", self.lda, K), ("B", self.ldb, N), ("C", self.ldc, N)):
                sizes = rows.astype(np.int64) * cols
                offs = np.concatenate([[0], np.cumsum(sizes)[:-1]])
                flat = torch.randn(int(sizes.sum()), dtype=torch.float64, device=dev, generator=g).to(dt)
                esz = flat.element_size()
                ptrs = flat.data_ptr() + torch.from_numpy(offs * esz).to(dev)
                parts[name] = (flat, ptrs, offs, sizes)
            self.bufs[tag] = parts
        self.C0 = {t: self.bufs[t]["C"][0].clone() for t in "ds"}
        ints = lambda v: torch.from_numpy(np.concatenate([v, [0]]).astype(np.int32)).to(dev)
        self.dM, self.dN, self.dK = ints(M), ints(N), ints(K)
        self.dla, self.dlb, self.dlc = ints(self.lda), ints(self.ldb), ints(self.ldc)
        self.l2 = f"A+B+C {self.bytes64 / 2**30:.2f} GiB (FP64) > L2 (126 MB)"

    def units(self):
        return self.flops / 1e9

    def config_extra(self):
        return {"M": "U{8..128}", "N": "U{8..128}", "K": "U{8..128}", "ld": "roundup(rows, 8)",
                "alpha": 1.0, "beta": 0.5, "gflop_per_step": self.flops / 1e9}

    def launches_per_step(self):
        return 1 + 4   # bucketize by max(M, N), then one launch per size bucket (four below 128)

    def _call(self, q, tag):
        b = self.bufs[tag]
        fn = q.lib.magmablas_dgemm_vbatched_max_nocheck if tag == "d" else q.lib.magmablas_sgemm_vbatched_max_nocheck
        fn(111, 111, vp(self.dM), vp(self.dN), vp(self.dK), 1.0, vp(b["A"][1]), vp(self.dla), vp(b["B"][1]),
           vp(self.dlb), 0.5, vp(b["C"][1]), vp(self.dlc), self.batch, 128, 128, 128, q.handle)
        return 0

    def restore(self, i):
        self.bufs["d"]["C"][0].copy_(self.C0["d"])

    def step(self, q, i):
        return self._call(q, "d")

    def restore_alt(self, i):
        self.bufs["s"]["C"][0].copy_(self.C0["s"])

    def step_alt(self, q, i):
        return self._call(q, "s")

    def ratios(self, value, alt_value):
        return {"fp32_over_fp64": alt_value / value}

    def _check(self, q, tag, sample):
        t = self.torch
        b = self.bufs[tag]
        b["C"][0].copy_(self.C0[tag])
        self._call(q, tag)
        q.sync()
        worst = 0.0
        for i in sample:
            m, n, k = int(self.M[i]), int(self.N[i]), int(self.K[i])
            sl = lambda nm, rows, cols: b[nm][0][int(b[nm][2][i]):int(b[nm][2][i]) + rows * cols].view(cols, rows)
            A = sl("A", int(self.lda[i]), k)[:, :m].T.double()
            Bm = sl("B", int(self.ldb[i]), n)[:, :k].T.double()
            C0 = self.C0[tag][int(b["C"][2][i]):int(b["C"][2][i]) + int(self.ldc[i]) * n].view(n, -1)[:, :m].T.double()
            C = sl("C", int(self.ldc[i]), n)[:, :m].T.double()
            ref = A @ Bm + 0.5 * C0
            # normalised max error |C - C_ref| / (k |A|max |B|max + beta |C0|max)
            err = (C - ref).abs().max() / ((A.abs().max() * Bm.abs().max() * k + 0.5 * C0.abs().max()) + 1e-300)
            worst = max(worst, float(err))
        b["C"][0].copy_(self.C0[tag])
        return worst

    def validate(self, q):
        sample = list(range(0, self.batch, max(1, self.batch // 200)))
        return {"gemm_err_max_fp64": self._check(q, "d", sample), "gemm_err_max_fp32": self._check(q, "s", sample)}

    def dominant_kernel(self, q, stream, reps=20):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        return {"kernel": "gemm_dmma_async_kernel (magmablas_dgemm_vbatched_max_nocheck: the FP64 tensor-core tile for "
                          "max(M,N) > 32, CUDA-core tiles below)", "ms": ms,
                "alg_bytes": self.bytes64, "tflops": self.flops / ms / 1e9}

    def e2e_setup(self):
        t = self.torch
        b = self.bufs["d"]
        self.h = {k: b[k][0].cpu().pin_memory() for k in "ABC"}
        self.hC0 = self.C0["d"].cpu().pin_memory()
        self.h2d = sum(self.h[k].numel() * 8 for k in "ABC")
        self.d2h = self.h["C"].numel() * 8

    def e2e_step(self, q, i):
        b = self.bufs["d"]
        b["A"][0].copy_(self.h["A"], non_blocking=True)
        b["B"][0].copy_(self.h["B"], non_blocking=True)
        b["C"][0].copy_(self.hC0, non_blocking=True)
        self.step(q, i)
        self.h["C"].copy_(b["C"][0], non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None, sample=2000):
        import numpy as np

        import oracle

        b = self.bufs["d"]
        flat = {k: b[k][0][: int(b[k][2][sample - 1] + b[k][3][sample - 1])].cpu().numpy() for k in "ABC"}
        cols = {"A": self.K, "B": self.N, "C": self.N}
        rows = {"A": self.lda, "B": self.ldb, "C": self.ldc}
        mats = {k: [flat[k][int(b[k][2][i]):int(b[k][2][i] + b[k][3][i])].reshape(int(cols[k][i]), int(rows[k][i]))
                    for i in range(sample)] for k in "ABC"}
        fl = float((2.0 * self.M[:sample].astype(np.float64) * self.N[:sample] * self.K[:sample]).sum())
        done, t_total = 0.0, 0.0
        while t_total < seconds:
            t0 = time.perf_counter()
            oracle.lapack_gemm_vbatched(0, 0, self.M[:sample], self.N[:sample], self.K[:sample], 1.0, mats["A"],
                                        self.lda[:sample], mats["B"], self.ldb[:sample], 0.5, mats["C"],
                                        self.ldc[:sample], nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += fl
        return done / 1e9 / t_total, done, (nthreads or oracle.max_threads()), \
            f"{sample}-instance slices of the same inputs, re-run; dgemm (OpenBLAS 0.3.30, scipy) in an OpenMP " \
            f"loop, 1 BLAS thread each"


class TrsmVbatched:
    """magmablas_dtrsm_vbatched (Left, Lower, NoTrans, NonUnit) on 20,000 instances with
    M, N ~ U{8..128}, beside magmablas_dtrmm_vbatched on the same operands."""
    unit = "GFLOP/s"
    dtype = "f64"
    metric = "trsm_vbatched GFLOP/s (FP64; trmm_vbatched beside)"
    data = "synthetic: M, N ~ U{8..128} (splitmix64), A = N(0,1)/sqrt(m) + 2 I, B ~ N(0,1) (seeded)"
    alt_name = "trmm"

    def __init__(self, dev, batch=20000, seed=12):
        import numpy as np
        import torch

        from magma_b200 import testing as T

        self.torch, self.dev, self.batch = torch, dev, batch
        self.name = f"trsm_vbatched_{batch}_MN8-128_left_lower_notrans"
        M, N, _ = T.gemm_sizes(batch, 8, 128, seed=seed)
        r8 = lambda v: ((v + 7) // 8) * 8
        self.M, self.N = M, N
        self.lda, self.ldb = r8(M), r8(M)
        m64 = M.astype(np.float64)
        self.flops = float((m64 * m64 * N).sum())
        self.bytes64 = float(8 * (m64 * (m64 + 1) / 2 + 2 * m64 * N).sum())
        rng = np.random.default_rng(seed)
        sa = self.lda.astype(np.int64) * M
        sb = self.ldb.astype(np.int64) * N
        self.offa = np.concatenate([[0], np.cumsum(sa)[:-1]])
        self.offb = np.concatenate([[0], np.cumsum(sb)[:-1]])
        fa = rng.standard_normal(int(sa.sum()))
        for i in range(batch):
            m, la = int(M[i]), int(self.lda[i])
            blk = fa[self.offa[i]:self.offa[i] + la * m].reshape(m, la)
            blk *= 1.0 / np.sqrt(m)
            blk[np.arange(m), np.arange(m)] += 2.0
        fb = rng.standard_normal(int(sb.sum()))
        self.hA, self.hB0 = fa, fb
        self.A = torch.from_numpy(fa).to(dev)
        self.B0 = torch.from_numpy(fb).to(dev)
        self.B = self.B0.clone()
        self.pA = self.A.data_ptr() + torch.from_numpy(self.offa * 8).to(dev)
        self.pB = self.B.data_ptr() + torch.from_numpy(self.offb * 8).to(dev)
        ints = lambda v: torch.from_numpy(np.concatenate([v, [0]]).astype(np.int32)).to(dev)
        self.dM, self.dN, self.dla, self.dlb = ints(M), ints(N), ints(self.lda), ints(self.ldb)
        self.l2 = f"A+B {self.bytes64 / 2**30:.2f} GiB (FP64 triangle + B read and written) > L2; B restored between steps"

    def units(self):
        return self.flops / 1e9

    def config_extra(self):
        return {"M": "U{8..128}", "N": "U{8..128}", "ld": "roundup(M, 8)", "side": "left", "uplo": "lower",
                "trans": "no", "diag": "non-unit", "alpha": 1.0, "gflop_per_step": self.flops / 1e9}

    def launches_per_step(self):
        return 1

    def _call(self, q, fn):
        fn(141, 122, 111, 131, vp(self.dM), vp(self.dN), 1.0, vp(self.pA), vp(self.dla), vp(self.pB), vp(self.dlb),
           self.batch, 128, 128, q.handle)
        return 0

    def restore(self, i):
        self.B.copy_(self.B0)

    restore_alt = restore

    def step(self, q, i):
        return self._call(q, q.lib.magmablas_dtrsm_vbatched_max_nocheck)

    def step_alt(self, q, i):
        return self._call(q, q.lib.magmablas_dtrmm_vbatched_max_nocheck)

    def ratios(self, value, alt_value):
        return {"trmm_over_trsm": alt_value / value}

    def validate(self, q):
        import numpy as np

        import oracle

        out = {}
        for tag, fn in (("trsm", self.step), ("trmm", self.step_alt)):
            self.restore(0)
            fn(q, 0)
            q.sync()
            got = self.B.cpu().numpy()
            worst = 0.0
            for i in range(0, self.batch, max(1, self.batch // 100)):
                m, n, la, lb = int(self.M[i]), int(self.N[i]), int(self.lda[i]), int(self.ldb[i])
                A = self.hA[self.offa[i]:self.offa[i] + la * m].reshape(m, la).copy()
                ref = self.hB0[self.offb[i]:self.offb[i] + lb * n].reshape(n, lb).copy()
                oracle.dtri(tag == "trsm", True, True, False, False, m, n, 1.0, A, ref)
                g = got[self.offb[i]:self.offb[i] + lb * n].reshape(n, lb)
                worst = max(worst, float(np.abs(g - ref).max()))
            out[f"max_abs_diff_vs_oracle_{tag}"] = worst
        self.restore(0)
        return out

    def dominant_kernel(self, q, stream, reps=20):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        return {"kernel": "tri_panel_kernel<double,solve> (magmablas_dtrsm_vbatched_max_nocheck)", "ms": ms,
                "alg_bytes": self.bytes64, "tflops": self.flops / ms / 1e9}

    def e2e_setup(self):
        t = self.torch
        self.hAp = t.from_numpy(self.hA).pin_memory()
        self.hBp = t.from_numpy(self.hB0).pin_memory()
        self.hX = t.empty_like(self.hBp).pin_memory()
        self.h2d = self.hAp.numel() * 8 + self.hBp.numel() * 8
        self.d2h = self.hX.numel() * 8

    def e2e_step(self, q, i):
        self.A.copy_(self.hAp, non_blocking=True)
        self.B.copy_(self.hBp, non_blocking=True)
        self.step(q, i)
        self.hX.copy_(self.B, non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None, sample=4000):
        import numpy as np

        import oracle

        As = [self.hA[self.offa[i]:self.offa[i] + int(self.lda[i] * self.M[i])].reshape(int(self.M[i]),
                                                                                     int(self.lda[i]))
              for i in range(sample)]
        fl = float((self.M[:sample].astype(np.float64) ** 2 * self.N[:sample]).sum())
        done, t_total = 0.0, 0.0
        while t_total < seconds:
            Bs = [self.hB0[self.offb[i]:self.offb[i] + int(self.ldb[i] * self.N[i])].reshape(int(self.N[i]),
                                                                                         int(self.ldb[i])).copy()
                  for i in range(sample)]
            t0 = time.perf_counter()
            oracle.lapack_dtri_vbatched(True, True, True, False, False, self.M[:sample], self.N[:sample], 1.0, As,
                                        self.lda[:sample], Bs, self.ldb[:sample], nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += fl
        return done / 1e9 / t_total, done, (nthreads or oracle.max_threads()), \
            f"{sample}-instance slices of the same inputs, re-run; dtrsm (OpenBLAS 0.3.30, scipy) in an OpenMP " \
            f"loop, 1 BLAS thread each"


class C4CholVbatched:
    """Variable-size Cholesky solve on 50,000 SPD instances, n power-law on [4, 512] (exponent -1.5),
    1-8 RHS: magma_dposv_vbatched_max_nocheck (FP64) replayed as one captured CUDA graph, beside
    magma_dsposv_vbatched_max_nocheck (FP32 factor + FP64 refinement), also graph-replayed."""
    unit = "solves/s"
    dtype = "f64"
    metric = "vbatched Cholesky solves/s at bwd err <=1e-14 (FP64; FP32-factor + FP64-refinement beside)"
    data = "synthetic: n ~ power law on [4,512] (inverse CDF, seeded), A = G G^T + n I with G ~ N(0,1), B ~ N(0,1)"
    alt_name = "mixed"

    def __init__(self, dev, batch=50000, seed=4):
        import numpy as np
        import torch

        self.torch, self.dev, self.batch = torch, dev, batch
        self.name = f"c4_posv_vbatched_{batch}_n4-512_powerlaw1.5_nrhs1-8"
        rng = np.random.default_rng(seed)
        a, b = 4.0 ** -0.5, 512.0 ** -0.5
        u = rng.random(batch)
        n = np.rint((a - u * (a - b)) ** -2.0).astype(np.int64).clip(4, 512)
        nrhs = rng.integers(1, 9, batch)
        self.n, self.nrhs = n, nrhs
        pad = lambda v: ((v + 3) // 4) * 4
        order = np.argsort(n, kind="stable")            # lay instances out grouped by size
        szA, szB = pad(n * n), pad(n * nrhs)
        offA = np.zeros(batch, np.int64)
        offB = np.zeros(batch, np.int64)
        offA[order] = np.concatenate([[0], np.cumsum(szA[order])[:-1]])
        offB[order] = np.concatenate([[0], np.cumsum(szB[order])[:-1]])
        self.offA, self.offB = offA, offB
        self.A0 = torch.zeros(int(szA.sum()), dtype=torch.float64, device=dev)
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        for nv in np.unique(n):
            ids = np.nonzero(n == nv)[0]
            nv = int(nv)
            G = torch.randn(len(ids), nv, nv, dtype=torch.float64, device=dev, generator=g)
            S = G @ G.transpose(1, 2) + nv * torch.eye(nv, dtype=torch.float64, device=dev)
            idx = torch.from_numpy(offA[ids]).to(dev)[:, None] + torch.arange(nv * nv, device=dev)[None, :]
            self.A0[idx.reshape(-1)] = S.reshape(-1)
            del G, S, idx
        self.B0 = torch.randn(int(szB.sum()), dtype=torch.float64, device=dev, generator=g)
        self.A = self.A0.clone()
        self.B = self.B0.clone()
        self.X = torch.zeros_like(self.B0)
        self.Am = self.A0.clone()
        self.W = torch.empty(int(pad(n * (n + nrhs)).sum()), dtype=torch.float32, device=dev)
        offW = np.concatenate([[0], np.cumsum(pad(n * (n + nrhs)))[:-1]])
        P = lambda buf, off, esz: buf.data_ptr() + torch.from_numpy(off * esz).to(dev)
        self.pA, self.pB, self.pX = P(self.A, offA, 8), P(self.B, offB, 8), P(self.X, offB, 8)
        self.pAm, self.pW = P(self.Am, offA, 8), P(self.W, offW, 4)
        self.pB0 = P(self.B0, offB, 8)   # the mixed arm reads B0 (dsposv leaves B untouched)
        ints = lambda v: torch.from_numpy(np.concatenate([v, [0]]).astype(np.int32)).to(dev)
        self.dn, self.dr = ints(n), ints(nrhs)
        self.info = torch.zeros(batch + 1, dtype=torch.int32, device=dev)
        self.it = torch.zeros(batch + 1, dtype=torch.int32, device=dev)
        self.flops = float((n ** 3 / 3.0 + n ** 2 / 2.0 + n / 6.0 + 2.0 * n * n * nrhs).sum())
        self.l2 = f"A {self.A0.numel() * 8 / 2**30:.2f} GiB > L2 (126 MB)"
        self.graphs = {}

    def units(self):
        return self.batch

    def config_extra(self):
        return {"n": "power law on [4,512], exponent -1.5", "nrhs": "U{1..8}", "uplo": "lower",
                "graph": "one captured CUDA graph per step", "gflop_per_step": self.flops / 1e9}

    def launches_per_step(self):
        # bucketize + largest-first sort, then the persistent queue kernel (tuning value 19 = 1)
        # or the per-bucket kernels of orders <= 512: factor + solve fused for n <= 64 (4
        # buckets), separate for the 3 blocked buckets
        from magma_b200 import _lib
        lib = _lib.load()
        count = lib.magma_b200_tuning_get(None, 0)
        vals = (C.c_int * count)()
        queue = lib.magma_b200_tuning_get(vals, count) == count and vals[19] == 1
        return 2 + (1 if queue else 4 + 3 * 2)

    def _raw_fp64(self, q):
        return q.lib.magma_dposv_vbatched_max_nocheck(122, vp(self.dn), vp(self.dr), vp(self.pA), vp(self.dn),
                                                      vp(self.pB), vp(self.dn), vp(self.info), self.batch, 512, 8,
                                                      q.handle)

    def _raw_mixed(self, q):
        return q.lib.magma_dsposv_vbatched_max_nocheck(122, vp(self.dn), vp(self.dr), vp(self.pAm), vp(self.dn),
                                                       vp(self.pB0), vp(self.dn), vp(self.pX), vp(self.dn),
                                                       vp(self.pW), vp(self.it), vp(self.info), self.batch, 512, 8,
                                                       q.handle)

    def _graph(self, q, key, fn):
        """Capture fn once into a CUDA graph on the queue's stream (after an eager call has
        grown the queue workspace to its final size), then replay it."""
        t = self.torch
        if key not in self.graphs:
            assert fn(q) == 0
            t.cuda.synchronize()
            g = t.cuda.CUDAGraph()
            with t.cuda.graph(g, stream=t.cuda.current_stream()):
                rc = fn(q)
            assert rc == 0, rc
            self.graphs[key] = g
        self.graphs[key].replay()
        return 0

    def restore(self, i):
        self.A.copy_(self.A0)
        self.B.copy_(self.B0)

    def step(self, q, i):
        return self._graph(q, "fp64", self._raw_fp64)

    def restore_alt(self, i):
        self.Am.copy_(self.A0)

    def step_alt(self, q, i):
        return self._graph(q, "mixed", self._raw_mixed)

    def ratios(self, value, alt_value):
        return {"mixed_over_fp64": alt_value / value}

    def _bwd(self, X, sample):
        import numpy as np

        A0, B0 = self.A0.cpu().numpy(), self.B0.cpu().numpy()
        Xh = X.cpu().numpy()
        worst = 0.0
        for i in sample:
            n, r = int(self.n[i]), int(self.nrhs[i])
            A = A0[self.offA[i]:self.offA[i] + n * n].reshape(n, n)
            B = B0[self.offB[i]:self.offB[i] + n * r].reshape(r, n).T
            x = Xh[self.offB[i]:self.offB[i] + n * r].reshape(r, n).T
            R = B - A @ x
            den = np.abs(A).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(B).max(axis=0)
            worst = max(worst, float((np.abs(R).max(axis=0) / den).max()))
        return worst

    def validate(self, q):
        import numpy as np

        t = self.torch
        sample = sorted(set(np.argsort(self.n)[-50:].tolist() + list(range(0, self.batch, self.batch // 250))))
        self.restore(0)
        assert self._raw_fp64(q) == 0
        q.sync()
        be64 = self._bwd(self.B, sample)
        nz64 = int((self.info[:self.batch] != 0).sum())
        self.restore_alt(0)
        assert self._raw_mixed(q) == 0
        q.sync()
        bem = self._bwd(self.X, sample)
        it = self.it[:self.batch].cpu()
        hist = {int(k): int(v) for k, v in zip(*t.unique(it, return_counts=True))}
        self.restore(0)
        return {"bwd_err_max_fp64": be64, "bwd_err_max_mixed": bem, "iter_hist_mixed": hist, "info_nonzero": nz64,
                "bwd_err_sample": len(sample)}

    def _bwd_all(self, X):
        from magma_b200.testing import backward_error_vbatched_torch

        return backward_error_vbatched_torch(self.A0, X, self.B0, self.n, self.nrhs, self.offA, self.offB)

    def check_last(self, q):
        """The bar on the last timed FP64 step's outputs (B overwritten by X, info), every instance."""
        q.sync()
        return accuracy_gate("last_step_fp64", self._bwd_all(self.B), self.info[:self.batch])

    def check_last_alt(self, q):
        """The bar on the last timed mixed step's outputs (X, info), every instance."""
        q.sync()
        return accuracy_gate("last_step_mixed", self._bwd_all(self.X), self.info[:self.batch])

    def dominant_kernel(self, q, stream, reps=5):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        alg = float((16.0 * self.n ** 2 + 16.0 * self.n * self.nrhs + 4).sum())
        name = ("chol_queue_kernel<double,1,1,8> (posv_vbatched: one persistent launch after bucketize + sort)"
                if self.launches_per_step() == 3 else "posv_vbatched (graph: potrf/potrs bucket kernels)")
        return {"kernel": name, "ms": ms, "alg_bytes": alg, "tflops": self.flops / ms / 1e9}

    def extras(self, q, stream, reps=3):
        """Per-bucket roofline: each size bucket's instances solved alone (eager calls on a
        sub-batch of the same pointers), FP64 flops against the nominal FP64 peak and
        compulsory bytes against the measured copy bandwidth."""
        import numpy as np

        t = self.torch
        peaks = measured_peaks()
        out = []
        edges = [(4, 32), (33, 64), (65, 128), (129, 256), (257, 512)]
        ints = lambda v: t.from_numpy(np.concatenate([v, [0]]).astype(np.int32)).to(self.dev)
        for lo, hi in edges:
            ids = np.nonzero((self.n >= lo) & (self.n <= hi))[0]
            if len(ids) == 0:
                continue
            sel = t.from_numpy(ids).to(self.dev)
            pA, pB = self.pA[sel].contiguous(), self.pB[sel].contiguous()
            dn, dr = ints(self.n[ids]), ints(self.nrhs[ids])
            info = t.zeros(len(ids) + 1, dtype=t.int32, device=self.dev)
            mx_n, mx_r = int(self.n[ids].max()), int(self.nrhs[ids].max())
            call = lambda i: q.lib.magma_dposv_vbatched_max_nocheck(122, vp(dn), vp(dr), vp(pA), vp(dn), vp(pB),
                                                                    vp(dn), vp(info), len(ids), mx_n, mx_r,
                                                                    q.handle)
            self.restore(0)
            call(0)
            ms = timed_restore(stream, call, self.restore, reps) / reps
            nv, rv = self.n[ids].astype(np.float64), self.nrhs[ids]
            fl = float((nv ** 3 / 3.0 + nv ** 2 / 2.0 + nv / 6.0 + 2.0 * nv * nv * rv).sum())
            by = float((16.0 * nv ** 2 + 16.0 * nv * rv + 4).sum())
            tf, gbs = fl / (ms * 1e-3) / 1e12, by / (ms * 1e-3) / 1e9
            out.append({"n": f"[{lo},{hi}]", "count": int(len(ids)), "ms": ms, "tflops": tf,
                        "fp64_frac_nominal": tf / FP64_NOMINAL_TFLOPS, "gbs": gbs,
                        "hbm_frac": gbs / peaks["hbm_gbs"], "flop_per_byte": fl / by})
        self.restore(0)
        return {"per_bucket": out}

    def e2e_setup(self):
        self.hA = self.A0.cpu().pin_memory()
        self.hB = self.B0.cpu().pin_memory()
        self.hX = self.torch.empty_like(self.hB).pin_memory()
        self.hI = self.torch.empty(self.batch + 1, dtype=self.torch.int32).pin_memory()
        self.h2d = (self.hA.numel() + self.hB.numel()) * 8
        self.d2h = self.hX.numel() * 8 + self.hI.numel() * 4

    def e2e_step(self, q, i):
        self.A.copy_(self.hA, non_blocking=True)
        self.B.copy_(self.hB, non_blocking=True)
        self.step(q, i)
        self.hX.copy_(self.B, non_blocking=True)
        self.hI.copy_(self.info, non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None, sample=5000):
        import oracle

        A0, B0 = self.A0.cpu().numpy(), self.B0.cpu().numpy()
        n, r = self.n[:sample], self.nrhs[:sample]
        done, t_total = 0, 0.0
        while t_total < seconds:
            As = [A0[self.offA[i]:self.offA[i] + n[i] * n[i]].reshape(n[i], n[i]).copy() for i in range(sample)]
            Bs = [B0[self.offB[i]:self.offB[i] + n[i] * r[i]].reshape(r[i], n[i]).copy() for i in range(sample)]
            t0 = time.perf_counter()
            oracle.lapack_dposv_vbatched(As, Bs, n, r, n, n, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += sample
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} solves (first {sample} instances, re-run); LAPACK dpotrf + dpotrs (OpenBLAS 0.3.30, scipy) " \
            f"in an OpenMP loop, 1 BLAS thread each"

class QrBatched:
    """Householder QR, 10,000 x (64x64) (magma_dgeqrf_batched)."""
    name = "qr_dgeqrf_batched_10000x64x64"
    unit = "factorizations/s"
    dtype = "f64"
    metric = "dgeqrf_batched factorizations/s (FP64)"
    data = "synthetic: seeded U[-1,1] (splitmix64)"

    def __init__(self, dev, batch=10000, m=64, n=64, seed=6):
        import torch

        from magma_b200 import testing as T
        from magma_b200.api import ptr_array

        self.torch, self.dev, self.batch, self.m, self.n = torch, dev, batch, m, n
        self.A_np, _ = T.lu_uniform(batch, n, 1, seed=seed)
        self.A0 = torch.from_numpy(self.A_np).to(dev)
        self.A = torch.empty_like(self.A0)
        self.tau = torch.zeros((batch, n), dtype=torch.float64, device=dev)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.pA, self.pT = ptr_array(self.A), ptr_array(self.tau)
        self.l2 = f"A ({8 * batch * m * n / 2**20:.0f} MiB) > L2, restored from a device copy between steps"

    def units(self):
        return self.batch

    def config_extra(self):
        return {"m": self.m, "n": self.n}

    def bytes_per_unit(self):
        return 2 * 8 * self.m * self.n + 8 * self.n

    def flops_per_unit(self):
        m, n = self.m, self.n
        return 2 * m * n * n - 2 * n ** 3 / 3

    def launches_per_step(self):
        return 1

    def restore(self, i):
        self.A.copy_(self.A0)

    def step(self, q, i):
        return q.lib.magma_dgeqrf_batched(self.m, self.n, vp(self.pA), self.m, vp(self.pT), vp(self.info),
                                          self.batch, q.handle)

    def validate(self, q):
        import oracle

        self.restore(0)
        self.step(q, 0)
        q.sync()
        k = 256
        G = self.A[:k].cpu().numpy()
        O = self.A_np[:k].copy()
        tau_o = oracle.dgeqrf_batched(O, self.m)
        return {"max_abs_diff_vs_oracle": float(abs(G - O).max()),
                "tau_max_abs_diff_vs_oracle": float(abs(self.tau[:k].cpu().numpy() - tau_o).max())}

    def dominant_kernel(self, q, stream, reps=50):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        fl = self.flops_per_unit() * self.batch
        return {"kernel": "geqrf_lanes_kernel<16,4,64>", "ms": ms, "alg_bytes": self.bytes_per_unit() * self.batch,
                "tflops": fl / (ms * 1e-3) / 1e12,
                "alg_note": f"FP64 {fl / (ms * 1e-3) / 1e12:.2f} TFLOP/s of {FP64_NOMINAL_TFLOPS} nominal"}

    def e2e_setup(self):
        t = self.torch
        self.hA = t.from_numpy(self.A_np).pin_memory()
        self.hR = t.empty_like(self.hA).pin_memory()
        self.hT = t.empty((self.batch, self.n), dtype=t.float64).pin_memory()
        self.h2d = self.hA.numel() * 8
        self.d2h = self.hR.numel() * 8 + self.hT.numel() * 8

    def e2e_step(self, q, i):
        self.A.copy_(self.hA, non_blocking=True)
        self.step(q, i)
        self.hR.copy_(self.A, non_blocking=True)
        self.hT.copy_(self.tau, non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None):
        import oracle

        done, t_total = 0, 0.0
        while t_total < seconds:
            A = self.A_np.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgeqrf_batched(A, self.m, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += self.batch
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} factorizations (10,000-instance batches, same inputs); LAPACK dgeqrf (OpenBLAS 0.3.30, " \
            f"scipy) in an OpenMP loop, 1 BLAS thread each"



class _Flush:
    """Writes a buffer larger than L2 (outside the timed brackets) so a restored input
    that fits in L2 is read from HBM by the timed step."""

    def __init__(self, torch, dev):
        self.buf = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def __call__(self):
        self.buf.zero_()


class GetriBatched:
    """LU + out-of-place inverse, 10,000 x (32x32) (magma_dgetrf_batched +
    magma_dgetri_outofplace_batched, timed together as testing_zgetri_batched.cpp:119-122)."""
    name = "getri_dgetrf+dgetri_outofplace_batched_10000x32"
    unit = "inverses/s"
    dtype = "f64"
    metric = "getrf + getri_outofplace inverses/s (FP64)"
    data = "synthetic: seeded U[-1,1] (splitmix64)"

    def __init__(self, dev, batch=10000, n=32, seed=8):
        import torch

        from magma_b200 import testing as T
        from magma_b200.api import ptr_array

        self.torch, self.dev, self.batch, self.n = torch, dev, batch, n
        self.A_np, _ = T.lu_uniform(batch, n, 1, seed=seed)
        self.A0 = torch.from_numpy(self.A_np).to(dev)
        self.A = torch.empty_like(self.A0)
        self.inv = torch.empty_like(self.A0)
        self.ipiv = torch.zeros((batch, n), dtype=torch.int32, device=dev)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.pA, self.pI, self.pP = ptr_array(self.A), ptr_array(self.inv), ptr_array(self.ipiv)
        self.flush = _Flush(torch, dev)
        self.l2 = "A restored, then a 252 MiB buffer written (L2 flushed) between steps"

    def units(self):
        return self.batch

    def config_extra(self):
        return {"n": self.n}

    def bytes_per_unit(self):
        n = self.n
        return 3 * 8 * n * n + 4 * n + 4        # read A, write LU and inv(A), pivots, info

    def launches_per_step(self):
        return 2                                # getrf, the fused inverse (n <= 32)

    def restore(self, i):
        self.A.copy_(self.A0)
        self.flush()

    def step(self, q, i):
        rc = q.lib.magma_dgetrf_batched(self.n, self.n, vp(self.pA), self.n, vp(self.pP), vp(self.info),
                                        self.batch, q.handle)
        return rc or q.lib.magma_dgetri_outofplace_batched(self.n, vp(self.pA), self.n, vp(self.pP), vp(self.pI),
                                                           self.n, vp(self.info), self.batch, q.handle)

    def validate(self, q):
        import numpy as np

        self.restore(0)
        self.step(q, 0)
        q.sync()
        k = 200
        X = self.inv[:k].cpu().numpy()
        res = max(float(np.abs(self.A_np[b].T @ X[b].T - np.eye(self.n)).max()) for b in range(k))
        return {"max_abs_A_invA_minus_I": res, "infos_nonzero": int((self.info != 0).sum())}

    def dominant_kernel(self, q, stream, reps=50):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        fl = 2 * self.n ** 3 * self.batch
        return {"kernel": "getrf+getri (getrf_small_kernel, getri_small_kernel)", "ms": ms,
                "alg_bytes": self.bytes_per_unit() * self.batch, "tflops": fl / (ms * 1e-3) / 1e12,
                "alg_note": "the whole step (2 launches); 2 n^3 flops per inverse"}

    def e2e_setup(self):
        t = self.torch
        self.hA = t.from_numpy(self.A_np).pin_memory()
        self.hX = t.empty_like(self.hA).pin_memory()
        self.hI = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.h2d = self.hA.numel() * 8
        self.d2h = self.hX.numel() * 8 + self.hI.numel() * 4

    def e2e_step(self, q, i):
        self.A.copy_(self.hA, non_blocking=True)
        self.step(q, i)
        self.hX.copy_(self.inv, non_blocking=True)
        self.hI.copy_(self.info, non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None):
        import oracle

        done, t_total = 0, 0.0
        while t_total < seconds:
            A = self.A_np.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgetri_batched(A, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += self.batch
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} inverses (10,000-instance batches, same inputs); LAPACK dgetrf + dgetri (OpenBLAS 0.3.30, " \
            f"scipy) in an OpenMP loop, 1 BLAS thread each"


class NopivBatched:
    """LU without pivoting + solve, 10,000 x (32x32), 1 RHS (magma_dgesv_nopiv_batched), with
    the random-butterfly solve (magma_dgesv_rbt_batched) on the same inputs as the second arm."""
    name = "nopiv_dgesv_nopiv_batched_10000x32_nrhs1"
    unit = "solves/s"
    dtype = "f64"
    metric = "gesv_nopiv_batched solves/s (FP64; gesv_rbt_batched beside)"
    data = "synthetic: seeded U[-1,1] (splitmix64) + 32 on the diagonal (no pivoting needed)"
    alt_name = "rbt"

    def __init__(self, dev, batch=10000, n=32, nrhs=1, seed=9):
        import torch

        from magma_b200 import testing as T
        from magma_b200.api import ptr_array

        self.torch, self.dev, self.batch, self.n, self.nrhs = torch, dev, batch, n, nrhs
        self.A_np, self.B_np = T.lu_uniform(batch, n, nrhs, seed=seed)
        for i in range(n):
            self.A_np[:, i, i] += n
        self.A0 = torch.from_numpy(self.A_np).to(dev)
        self.B0 = torch.from_numpy(self.B_np).to(dev)
        self.A, self.B = torch.empty_like(self.A0), torch.empty_like(self.B0)
        self.info = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.pA, self.pB = ptr_array(self.A), ptr_array(self.B)
        self.flush = _Flush(torch, dev)
        self.l2 = "A, B restored, then a 252 MiB buffer written (L2 flushed) between steps"

    def units(self):
        return self.batch

    def config_extra(self):
        return {"n": self.n, "nrhs": self.nrhs}

    def bytes_per_unit(self):
        n, r = self.n, self.nrhs
        return 2 * 8 * n * n + 2 * 8 * n * r + 4

    def launches_per_step(self):
        return 1

    def restore(self, i):
        self.A.copy_(self.A0)
        self.B.copy_(self.B0)
        self.flush()

    restore_alt = restore

    def step(self, q, i):
        return q.lib.magma_dgesv_nopiv_batched(self.n, self.nrhs, vp(self.pA), self.n, vp(self.pB), self.n,
                                               vp(self.info), self.batch, q.handle)

    def step_alt(self, q, i):
        return q.lib.magma_dgesv_rbt_batched(self.n, self.nrhs, vp(self.pA), self.n, vp(self.pB), self.n,
                                             vp(self.info), self.batch, q.handle)

    def ratios(self, value, alt_value):
        return {"rbt_over_nopiv": alt_value / value}

    def check_last(self, q, tag="last_step_nopiv"):
        """The bar on the last timed step's outputs (B overwritten by X, info), every instance."""
        from magma_b200.testing import backward_error_torch

        q.sync()
        return accuracy_gate(tag, backward_error_torch(self.A0, self.B, self.B0).amax(dim=1), self.info)

    def check_last_alt(self, q):
        return self.check_last(q, "last_step_rbt")

    def validate(self, q):
        from magma_b200 import testing as T

        out = {}
        for tag, fn in (("nopiv", self.step), ("rbt", self.step_alt)):
            self.restore(0)
            fn(q, 0)
            q.sync()
            out[f"bwd_err_max_{tag}"] = float(T.backward_error(self.A_np, self.B.cpu().numpy(), self.B_np,
                                                               self.n).max())
        return out

    def dominant_kernel(self, q, stream, reps=50):
        ms = timed_restore(stream, lambda i: self.step(q, i), self.restore, reps) / reps
        return {"kernel": "gesv_small_kernel<double,32,1,1> (no pivoting)", "ms": ms,
                "alg_bytes": self.bytes_per_unit() * self.batch, "tflops": None}

    def e2e_setup(self):
        t = self.torch
        self.hA = t.from_numpy(self.A_np).pin_memory()
        self.hB = t.from_numpy(self.B_np).pin_memory()
        self.hX = t.empty_like(self.hB).pin_memory()
        self.hI = t.empty(self.batch, dtype=t.int32).pin_memory()
        self.h2d = self.hA.numel() * 8 + self.hB.numel() * 8
        self.d2h = self.hX.numel() * 8 + self.hI.numel() * 4

    def e2e_step(self, q, i):
        self.A.copy_(self.hA, non_blocking=True)
        self.B.copy_(self.hB, non_blocking=True)
        self.step(q, i)
        self.hX.copy_(self.B, non_blocking=True)
        self.hI.copy_(self.info, non_blocking=True)

    def cpu_reference(self, seconds=10.0, nthreads=None):
        import oracle

        done, t_total = 0, 0.0
        while t_total < seconds:
            A, B = self.A_np.copy(), self.B_np.copy()
            t0 = time.perf_counter()
            oracle.lapack_dgesv_batched(A, B, nthreads=nthreads)
            t_total += time.perf_counter() - t0
            done += self.batch
        return done / t_total, done, (nthreads or oracle.max_threads()), \
            f"{done} solves (10,000-instance batches, same inputs); LAPACK dgesv (OpenBLAS 0.3.30, scipy; " \
            f"the CPU check of testing_zgesv_nopiv_batched.cpp) in an OpenMP loop, 1 BLAS thread each"


WORKLOADS = {"c3": C3Mixed, "c1": C1DgesvSmall, "c2": C2GemmVbatched, "c4": C4CholVbatched, "qr": QrBatched, "getri": GetriBatched,
             "nopiv": NopivBatched, "trsm": TrsmVbatched}
DEFAULT_STEPS = {"c3": (60, 5), "c1": (20000, 50), "c2": (50, 5), "c4": (20, 3), "c5": (10000, 200), "qr": (200, 5), "getri": (200, 5), "nopiv": (200, 5), "trsm": (50, 5)}


# ---------------------------------------------------------------------- main
def max_over_ranks(vals, dist, device=None):
    """Element-wise maximum of per-rank timings over all ranks (every rank receives the
    result); the job's time is its slowest replica's. `dist` None: one rank, unchanged."""
    if dist is None:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl != "reference":
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        return rank, world, local, dist
    return rank, world, local, None


def run_reference(args, rank):
    """The reference's CPU implementation (host LAPACK loop) on this host; rank 0 only."""
    if rank != 0:
        return
    import numpy as np

    import oracle
    from magma_b200 import testing as T

    nthreads = oracle.max_threads()
    if args.workload not in ("c1", "c2", "c3", "c4", "qr", "getri", "nopiv", "trsm"):
        print(json.dumps({"impl": "reference", "unavailable": "no reference arm for this workload (c5 is the "
                          "request loop; the reference has no serving front end)"}), flush=True)
        return
    metric, unit = METRIC, "solves/s"
    per_step = None          # units of work per step when they are not instances (GFLOP)
    # each step gets fresh copies of the inputs, made outside the timed call
    if args.workload == "c3":
        sample = 256
        A0, B0, _ = T.svd_logrand(sample, 256, 1e2, 1e6, nrhs=4, seed=3)
        prep = lambda: (A0.copy(), B0)   # noqa: E731
        fn = lambda a, b: oracle.lapack_dsgesv_batched(a, b, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (256x256, kappa in [1e2,1e6], 4 RHS); LAPACK dsgesv"
        cfg = {"workload": "c3_dsgesv_batched_2048x256_kappa1e2-1e6_nrhs4", "batch": sample, "n": 256, "nrhs": 4}
        dtype = C3Mixed.dtype
    elif args.workload in ("c2", "trsm"):
        # a bounded slice of the same size distribution, CPU-generated (same distributions)
        rng = np.random.default_rng(2)
        sample = 2000 if args.workload == "c2" else 4000
        if args.workload == "c2":
            M, N, K = (v[:sample] for v in T.gemm_sizes(20000, 8, 128, seed=2))
            r8 = lambda v: ((v + 7) // 8) * 8   # noqa: E731
            lda, ldb, ldc = r8(M), r8(K), r8(M)
            As = [rng.standard_normal((int(k), int(la))) for k, la in zip(K, lda)]
            Bs = [rng.standard_normal((int(nn), int(lb))) for nn, lb in zip(N, ldb)]
            Cs0 = [rng.standard_normal((int(nn), int(lc))) for nn, lc in zip(N, ldc)]
            prep = lambda: ([c.copy() for c in Cs0], None)   # noqa: E731
            fn = lambda cs, _: oracle.lapack_gemm_vbatched(0, 0, M, N, K, 1.0, As, lda, Bs, ldb, 0.5, cs, ldc,   # noqa: E731
                                                           nthreads=nthreads)
            per_step = float((2.0 * M.astype(np.float64) * N * K).sum()) / 1e9
            desc = f"{sample} instances per step (M, N, K ~ U{{8..128}}, alpha 1, beta 0.5); dgemm"
            cfg = {"workload": "c2_gemm_vbatched_20000_MNK8-128_alpha1_beta0.5", "batch": sample}
            dtype, metric, unit = C2GemmVbatched.dtype, C2GemmVbatched.metric, C2GemmVbatched.unit
        else:
            M, N, _ = (v[:sample] for v in T.gemm_sizes(20000, 8, 128, seed=12))
            r8 = lambda v: ((v + 7) // 8) * 8   # noqa: E731
            lda, ldb = r8(M), r8(M)
            As = []
            for m, la in zip(M, lda):
                a = rng.standard_normal((int(m), int(la))) / np.sqrt(float(m))
                a[np.arange(m), np.arange(m)] += 2.0
                As.append(a)
            Bs0 = [rng.standard_normal((int(nn), int(lb))) for nn, lb in zip(N, ldb)]
            prep = lambda: ([b.copy() for b in Bs0], None)   # noqa: E731
            fn = lambda bs, _: oracle.lapack_dtri_vbatched(True, True, True, False, False, M, N, 1.0, As, lda, bs,   # noqa: E731
                                                           ldb, nthreads=nthreads)
            per_step = float((M.astype(np.float64) ** 2 * N).sum()) / 1e9
            desc = f"{sample} instances per step (M, N ~ U{{8..128}}, left lower no-trans non-unit); dtrsm"
            cfg = {"workload": "trsm_vbatched_20000_MN8-128_left_lower_notrans", "batch": sample}
            dtype, metric, unit = TrsmVbatched.dtype, TrsmVbatched.metric, TrsmVbatched.unit
    elif args.workload == "c4":
        rng = np.random.default_rng(4)
        sample = 5000
        a_, b_ = 4.0 ** -0.5, 512.0 ** -0.5
        n = np.rint((a_ - rng.random(sample) * (a_ - b_)) ** -2.0).astype(np.int64).clip(4, 512)
        nr = rng.integers(1, 9, sample)
        As0 = []
        for nv in n:
            G = rng.standard_normal((int(nv), int(nv)))
            As0.append(G @ G.T + nv * np.eye(int(nv)))
        Bs0 = [rng.standard_normal((int(r), int(nv))) for nv, r in zip(n, nr)]
        prep = lambda: (([a.copy() for a in As0], [b.copy() for b in Bs0]), None)   # noqa: E731
        fn = lambda ab, _: oracle.lapack_dposv_vbatched(ab[0], ab[1], n, nr, n, n, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (SPD, n power law on [4,512], 1-8 RHS); dpotrf + dpotrs"
        cfg = {"workload": "c4_posv_vbatched_50000_n4-512_powerlaw1.5_nrhs1-8", "batch": sample}
        dtype, metric = C4CholVbatched.dtype, C4CholVbatched.metric
    elif args.workload == "getri":
        sample = 10000
        A0, _ = T.lu_uniform(sample, 32, 1, seed=8)
        prep = lambda: (A0.copy(), None)   # noqa: E731
        fn = lambda a, b: oracle.lapack_dgetri_batched(a, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (32x32); LAPACK dgetrf + dgetri"
        cfg = {"workload": GetriBatched.name, "batch": sample, "n": 32}
        dtype, metric, unit = GetriBatched.dtype, GetriBatched.metric, GetriBatched.unit
    elif args.workload == "nopiv":
        sample = 10000
        A0, B0 = T.lu_uniform(sample, 32, 1, seed=9)
        for i in range(32):
            A0[:, i, i] += 32
        prep = lambda: (A0.copy(), B0.copy())   # noqa: E731
        fn = lambda a, b: oracle.lapack_dgesv_batched(a, b, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (32x32 diagonally dominant, 1 RHS); LAPACK dgesv"
        cfg = {"workload": NopivBatched.name, "batch": sample, "n": 32, "nrhs": 1}
        dtype, metric, unit = NopivBatched.dtype, NopivBatched.metric, NopivBatched.unit
    elif args.workload == "qr":
        sample = 10000
        A0, _ = T.lu_uniform(sample, 64, 1, seed=6)
        prep = lambda: (A0.copy(), None)   # noqa: E731
        fn = lambda a, b: oracle.lapack_dgeqrf_batched(a, 64, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (64x64); LAPACK dgeqrf"
        cfg = {"workload": QrBatched.name, "batch": sample, "m": 64, "n": 64}
        dtype, metric, unit = QrBatched.dtype, QrBatched.metric, QrBatched.unit
    else:
        sample = 10000
        A0, B0 = T.lu_uniform(sample, 32, 1, seed=1)
        prep = lambda: (A0.copy(), B0.copy())   # noqa: E731
        fn = lambda a, b: oracle.lapack_dgesv_batched(a, b, nthreads=nthreads)   # noqa: E731
        desc = f"{sample} instances per step (32x32, 1 RHS); LAPACK dgesv"
        cfg = {"workload": C1DgesvSmall.name, "batch": sample, "n": 32, "nrhs": 1}
        dtype = C1DgesvSmall.dtype
    for _ in range(args.warmup):
        fn(*prep())
    times = []
    for _ in range(args.steps):
        a, b = prep()
        t0 = time.perf_counter()
        fn(a, b)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = (per_step if per_step is not None else sample) * args.steps / total
    del np
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": unit, "cores": nthreads, "kind": "reference",
                         "sample": desc + " (OpenBLAS 0.3.30, scipy) in an OpenMP loop, 1 BLAS thread each",
                         **host_cpu()},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)



def run_serving(args, rank, world):
    """C5: the request loop under Poisson arrivals (70% LU / 30% Cholesky, n log-uniform on
    [8, 1024], 1-16 RHS, 40 GB admission budget). A step is one request; each offered rate
    replays the same `steps` requests. Latency runs from a request's scheduled arrival to its
    result in host memory, on the host's monotonic clock."""
    import torch

    from magma_b200 import serve

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    reqs = serve.make_requests(args.steps, seed=5 + rank)
    warm = serve.make_requests(max(args.warmup, 3), seed=99 + rank)
    rates = [1e3, 3e3, 1e4, 3e4, 1e5]
    stated = 1e4
    sweep = []
    clocks = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(dev).uuid))
    with serve.Server(40 << 30, streams=6, max_batch=256) as sv:
        serve.run_load(sv, warm, rate=1e4, seed=1)
        clocks.start()
        for r in rates:
            res = serve.run_load(sv, reqs, rate=r, seed=int(r))
            sweep.append({k: res[k] for k in ("offered_rate", "throughput", "p50_ms", "p99_ms", "max_ms",
                                              "infos_nonzero", "max_submit_lag_ms")})
        clk = clocks.stop()
        stats = sv.stats()
    be = max(serve.backward_error(r) for r in reqs)
    at = next(x for x in sweep if x["offered_rate"] == stated)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([at["throughput"]], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        total = float(t.item())
    else:
        total = at["throughput"]
    if rank == 0:
        line = {
            "metric": "serving: requests/s with p50/p99 latency (arrival -> result on host)",
            "value": total, "unit": "requests/s", "n_gpus": world, "steps": args.steps, "warmup": len(warm),
            "ms_per_step": 1e3 / at["throughput"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": serve.__doc__.split("\n")[3].strip() + " (seeded)",
            "config": {"workload": f"c5_serving_{args.steps}req_lu70_chol30_n8-1024_nrhs1-16",
                       "offered_rate": stated, "hbm_budget_bytes": 40 << 30, "streams": 6, "max_batch": 256,
                       "parallelism": f"replicas x{world}", "l2": "per-request copies from pinned host memory"},
            "p50_ms": at["p50_ms"], "p99_ms": at["p99_ms"], "sweep": sweep, "bwd_err_max": be,
            "peak_device_bytes": stats["peak_bytes"], "micro_batches": stats["batches"],
            "e2e": {"value": total, "unit": "requests/s", "note": "every request is host-to-host",
                    "h2d_bytes_per_step": sum(8 * (r.A.size + r.B.size) for r in reqs) / len(reqs),
                    "d2h_bytes_per_step": sum(8 * r.X.size for r in reqs) / len(reqs)},
            "gpu_launches": None, "clocks": clk,
        }
        print(json.dumps(line), flush=True)

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["c5"], default="c3")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=None,
                    help="instances per GPU (default: the workload's own size; smaller only for profiling)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = DEFAULT_STEPS[args.workload][0] if args.impl == "ours" else 5
    if args.warmup is None:
        args.warmup = DEFAULT_STEPS[args.workload][1] if args.impl == "ours" else 3
    args.warmup = max(args.warmup, 3)

    rank, world, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "c5":
        run_serving(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import torch

    import magma_b200 as mb
    from magma_b200.api import Queue

    mb.load()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        W = WORKLOADS[args.workload](dev, **({"batch": args.batch} if args.batch else {}))
        q = Queue(stream, local)
        checks = W.validate(q)
        for i in range(args.warmup):
            if hasattr(W, "restore"):
                W.restore(i)
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
        rcs = []
        if hasattr(W, "restore"):
            ms_total = timed_restore(stream, lambda i: rcs.append(W.step(q, i)), W.restore, args.steps)
        else:
            ms_total = timed(stream, lambda i: rcs.append(W.step(q, i)), args.steps)
        if dist:
            dist.barrier()
        clk = clocks.stop()
        assert all(rc == 0 for rc in rcs), f"library returned {set(rcs)}"
        gate = {}
        gate_ok = all(v <= BWD_BAR for k, v in checks.items() if k.startswith("bwd_err_max"))
        if hasattr(W, "check_last"):
            g, ok = W.check_last(q)
            gate.update(g)
            gate_ok &= ok
        extra = {}
        if hasattr(W, "step_alt"):
            for i in range(3):
                W.restore_alt(i)
                W.step_alt(q, i)
            torch.cuda.synchronize(dev)
            ms_alt = timed_restore(stream, lambda i: W.step_alt(q, i), W.restore_alt, args.steps)
            extra["alt_ms_per_step"] = ms_alt / args.steps
            if hasattr(W, "check_last_alt"):
                g, ok = W.check_last_alt(q)
                gate.update(g)
                gate_ok &= ok
        dom = W.dominant_kernel(q, stream)
        extras = W.extras(q, stream) if hasattr(W, "extras") else {}
        # end to end (host buffers, copies inside each step)
        W.e2e_setup()
        ke = max(3, min(args.steps, 10 if args.workload == "c3" else 200))
        for i in range(2):
            W.e2e_step(q, i)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        ms_e2e = timed(stream, lambda i: W.e2e_step(q, i), ke)
    vals = max_over_ranks([ms_total, ms_e2e, extra.get("alt_ms_per_step", 0.0) * args.steps,
                           0.0 if gate_ok else 1.0], dist, dev)
    ms_total, ms_e2e, ms_alt_total, gate_failed = vals
    if gate_failed:
        # a step that missed the metric's accuracy bar has no throughput to report
        sys.stderr.write(f"bench: accuracy bar (backward error <= {BWD_BAR:g}, info == 0) missed on the last "
                         f"timed step: {json.dumps(gate)}\n")
        if dist:
            dist.destroy_process_group()
        sys.exit(3)
    units = W.units() * world
    value = units * args.steps / (ms_total * 1e-3)
    if rank == 0:
        peaks = measured_peaks()
        achieved = dom["alg_bytes"] / (dom["ms"] * 1e-3) / 1e9
        line = {
            "metric": getattr(W, "metric", METRIC), "value": value, "unit": W.unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": W.dtype, "data": W.data,
            "config": {"workload": W.name, "batch_per_gpu": W.batch, **W.config_extra(),
                       "parallelism": f"replicas x{world}", "l2": W.l2},
        }
        line.update(checks)
        line.update(gate)
        if gate:
            line["accuracy_gate"] = f"passed: every instance of the last timed step(s) at backward error <= {BWD_BAR:g}, info 0"
        line.update(extras)
        if ms_alt_total:
            alt_value = units * args.steps / (ms_alt_total * 1e-3)
            line[f"{W.alt_name}_value"] = alt_value
            line[f"{W.alt_name}_ms_per_step"] = ms_alt_total / args.steps
            line.update(W.ratios(value, alt_value))
        if "alg_flops" in dom:   # a tensor-core stage: quoted against the measured dense BF16 peak
            tf = dom["alg_flops"] / (dom["ms"] * 1e-3) / 1e12
            line["roofline"] = {
                "bound": "tensor", "achieved": tf, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                "frac": tf / peaks["bf16_tflops"], "traffic": profile_traffic(dom["kernel"].split(" ")[0], W.name),
                "kernel": dom["kernel"], "kernel_ms": dom["ms"], "alg_flops_per_launch": dom["alg_flops"],
                "peak_src": peaks["src"],
            }
        else:
            line["roofline"] = {
                "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": profile_traffic(dom["kernel"].split("<")[0].split(" ")[0], W.name),
                "kernel": dom["kernel"], "kernel_ms": dom["ms"], "alg_bytes_per_launch": dom["alg_bytes"],
                "peak_src": peaks["src"],
            }
        for key in ("stages", "alg_note"):
            if key in dom:
                line["roofline"][key] = dom[key]
        if dom.get("tflops"):
            line["roofline"]["kernel_tflops"] = dom["tflops"]
        line["e2e"] = {"value": units * ke / (ms_e2e * 1e-3), "unit": W.unit, "h2d_bytes_per_step": W.h2d,
                       "d2h_bytes_per_step": W.d2h, "steps": ke}
        if getattr(W, "e2e_api", None):
            line["e2e"]["api"] = W.e2e_api
        line["gpu_launches"] = args.steps * W.launches_per_step()
        line["clocks"] = clk
        if not args.no_cpu_baseline and world == 1:
            v, done, cores, sample = W.cpu_reference()
            line["cpu_baseline"] = {"value": v, "unit": W.unit, "cores": cores, "kind": "reference",
                                    "sample": sample, **host_cpu()}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
