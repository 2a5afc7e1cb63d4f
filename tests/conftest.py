import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def lu_golden():
    return np.load(GOLDEN / "lu_golden.npz")


@pytest.fixture(scope="session")
def chol_golden():
    return np.load(GOLDEN / "chol_golden.npz")


@pytest.fixture(scope="session")
def gemm_golden():
    return np.load(GOLDEN / "gemm_golden.npz")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for GPU tests. Fails (does not skip) when CUDA is absent:
    a GPU test that cannot reach the GPU must not pass."""
    import torch

    assert torch.cuda.is_available(), "GPU test selected but CUDA is not available"
    import magma_b200

    magma_b200.load()
    return torch.device("cuda", 0)
