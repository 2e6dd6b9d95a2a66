"""Shared test set-up: the `gpu` marker, golden fixtures and tolerances.

Tests marked ``gpu`` need a CUDA device (B200) and call the product library
through its C ABI; the others run on CPU only (oracle against the golden
fixtures, host logic, library loading and symbol export).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"

# tolerances (relative L2), from the parity targets of the hot path
TOL_FP64 = 1e-13   # FP64 Dslash vs the reference mult
TOL_FP32 = 1e-6    # FP32 Dslash
TOL_FP16 = 2e-3    # FP16 storage with FP32 arithmetic
TOL_SOL = 1e-8     # solutions vs the reference CG solution
TOL_RES = 1e-10    # true relative residual every solve must reach


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"ref_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def rel(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="session")
def port():
    import oracle
    return oracle.port()


@pytest.fixture(scope="session", params=["4x4x4x4", "6x2x4x4"])
def golden(request):
    return load_golden(request.param)


@pytest.fixture(scope="session")
def golden_full():
    return load_golden("4x4x4x4")
