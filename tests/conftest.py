import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the built libzogcu.so")
    config.addinivalue_line("markers", "slow: larger parity cases")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure; built on demand)."""
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def native():
    """libzogcu.so through its C ABI (ctypes).  GPU tests only."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from zog_b200 import _native
    from zog_b200 import build

    build.build()
    _native.load()
    return _native


def rel_l1(a, b):
    import numpy as np

    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).sum()
    num = np.abs(a - b).sum()
    return float(num / den) if den > 0 else float(num)
