import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def rel_l2(a, b):
    """||a - b|| / ||b|| over all entries (complex entries compared as complex numbers)."""
    a = np.asarray(a)
    b = np.asarray(b)
    dt = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a = a.astype(dt)
    b = b.astype(dt)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="session")
def golden_demo():
    return dict(np.load(os.path.join(GOLDEN, "demo_case.npz")))


@pytest.fixture(scope="session")
def golden_ops():
    return dict(np.load(os.path.join(GOLDEN, "operators_small.npz")))


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
