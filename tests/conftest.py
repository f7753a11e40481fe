import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: longer CPU pin (tens of seconds)")


def have_gpu():
    try:
        import ctypes

        rt = ctypes.CDLL("libcudart.so.12")
        n = ctypes.c_int(0)
        return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        try:
            import torch

            return torch.cuda.is_available()
        except Exception:
            return False


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture
def workdir(tmp_path):
    return str(tmp_path)
