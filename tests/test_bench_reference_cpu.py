"""bench.py's reference arm -- the reference's own CPU path for the workload (host LAPACK in
an OpenMP loop over instances) -- keeps the JSON contract of the bench line, and under
several ranks only rank 0 runs it. CPU only."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
ARGS = ["--impl", "reference", "--workload", "c1", "--steps", "1", "--warmup", "3"]


def run_bench(args, **env):
    return subprocess.run([sys.executable, "bench.py", *args], capture_output=True, text=True, cwd=ROOT,
                          env=dict(os.environ, **env), timeout=300)


def test_reference_arm_json_line():
    r = run_bench(ARGS)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "c1_dgesv_batched_10000x32_nrhs1"   # the same name as our arm's line
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_0_only():
    r = run_bench(ARGS, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_reference_arm_without_a_counterpart_says_unavailable():
    """The request loop (c5) has no reference implementation: one `unavailable` line, exit 0."""
    r = run_bench(["--impl", "reference", "--workload", "c5", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unavailable"]
