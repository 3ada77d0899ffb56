import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """The CUDA library on device 0.  Skips without a GPU; fails (does not
    skip) when a GPU is present but the library is missing."""
    if not has_cuda():
        pytest.skip("no CUDA device")
    import libnt_b200
    libnt_b200.lib()  # raises if the extension was not built
    return libnt_b200


@pytest.fixture
def rng():
    return np.random.default_rng(12345)


def rel_ok(v, v_ref, abs_terms, tol=1e-12):
    """Value parity for reductions in a different order:
    |v - v_ref| <= tol * sum|terms| per element (and exact where abs_terms == 0)."""
    v = np.asarray(v, np.float64)
    v_ref = np.asarray(v_ref, np.float64)
    bound = tol * np.asarray(abs_terms, np.float64)
    return np.all(np.abs(v - v_ref) <= bound)
