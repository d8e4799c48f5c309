import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def golden_sw():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "sw_golden.npz")))


@pytest.fixture(scope="session")
def golden_search():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "search_golden.npz")))
