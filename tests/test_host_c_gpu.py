"""A C program (tests/c/host_solve.c) calls the host-memory pipeline through the C ABI:
systems in page-locked host memory (magma_malloc_pinned), solved in chunks by
magma_b200_host_solve for the mixed-precision and the FP64 solver, checked on the host
(backward error <= 1e-14, info 0; the mixed solve refines, the FP64 solve keeps the
diagonal pivots of these diagonally dominant systems). The program is compiled here with
gcc against include/ and linked to the in-tree library."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")


def _build(tmp_path):
    exe = tmp_path / "host_solve"
    cmd = ["gcc", "-O2", "-std=c11", str(ROOT / "tests" / "c" / "host_solve.c"), f"-I{ROOT / 'include'}",
           f"-I{CUDA / 'include'}", f"-L{ROOT / 'magma_b200'}", "-lmagma_b200", f"-Wl,-rpath,{ROOT / 'magma_b200'}",
           "-lm", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_host_solve_c_program_compiles(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,batch,n", [(0, 300, 96), (0, 37, 256), (1, 300, 40), (1, 50, 130)])
def test_host_solve_c_program_runs(cuda, tmp_path, kind, batch, n):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), str(kind), str(batch), str(n)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    fields = r.stdout.split()
    assert fields[0] == "ok" and int(fields[1]) == kind and float(fields[4]) <= 1e-14
    if kind == 1:
        assert int(fields[5]) == batch * n   # every pivot on the diagonal
