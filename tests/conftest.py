import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native library")


def _has_gpu() -> bool:
    try:
        import ctypes
        cudart = ctypes.CDLL("libcudart.so.12")
    except OSError:
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False
    n = ctypes.c_int(0)
    return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


HAS_GPU = None


@pytest.fixture(scope="session")
def gpu_available():
    global HAS_GPU
    if HAS_GPU is None:
        HAS_GPU = _has_gpu()
    return HAS_GPU


def load_golden(name):
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", name))
