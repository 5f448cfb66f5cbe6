import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libdogcm_sht.so")


def pkg():
    return importlib.import_module("dennou-ogcm_b200")


def workloads():
    return importlib.import_module("dennou-ogcm_b200.workloads")


def relerr(a, b) -> float:
    """Largest per-field normwise relative error max|a-b| / max|b| (fields = leading axis)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim <= 1:
        a, b = a[None], b[None]
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    num = np.abs(a - b).max(axis=1)
    den = np.abs(b).max(axis=1)
    den = np.where(den == 0, 1.0, den)
    return float((num / den).max())


def load_golden(tag):
    return dict(np.load(os.path.join(GOLDEN, f"sht_{tag}.npz")))


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
