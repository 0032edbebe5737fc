import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libaifmm_b200.so")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


def _has_gpu() -> bool:
    import ctypes
    for name in ("libcuda.so.1", "libcuda.so"):
        try:
            cu = ctypes.CDLL(name)
        except OSError:
            continue
        n = ctypes.c_int(0)
        if cu.cuInit(0) != 0:
            return False
        return cu.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
