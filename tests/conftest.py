"""Shared pytest configuration: the `gpu` marker, library builds, scenario fixtures."""
import ctypes
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the CUDA library")


def _cuda_device_count() -> int:
    for name in ("libcudart.so", "libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"):
        try:
            rt = ctypes.CDLL(name)
        except OSError:
            continue
        n = ctypes.c_int(0)
        if rt.cudaGetDeviceCount(ctypes.byref(n)) == 0:
            return n.value
        return 0
    return 0


HAVE_GPU = _cuda_device_count() > 0


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def storm_lib():
    """The CUDA library, built in-tree if missing or stale (nvcc cross-compiles)."""
    from storm_b200 import build, fvt
    build.build()
    return fvt.lib()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle
