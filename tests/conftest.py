import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def cuda_device_count() -> int:
    """Device count from the CUDA runtime (no torch import needed)."""
    import ctypes
    try:
        rt = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            rt = ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")
        except OSError:
            return 0
    count = ctypes.c_int(0)
    if rt.cudaGetDeviceCount(ctypes.byref(count)) != 0:
        return 0
    return count.value


@pytest.fixture(scope="session")
def gpu():
    if cuda_device_count() < 1:
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return 0
