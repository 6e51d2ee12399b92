import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200 box)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def have_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not have_cuda():
        pytest.fail("this test needs a CUDA device")
    from cablegen_b200 import device
    device.init(0)
    return device
