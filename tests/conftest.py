import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libsph3.so")


@pytest.fixture(scope="session")
def oc():
    import oracle
    oracle.build()
    return oracle


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def golden():
    return load_golden


def rel_err(a, b, floor_frac=1e-6):
    """max |a - b| / max(|b|, floor_frac * rms(b)), elementwise over the array."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    rms = np.sqrt(np.mean(b * b))
    den = np.maximum(np.abs(b), floor_frac * rms + 1e-300)
    return float(np.max(np.abs(a - b) / den))
