"""pytest set-up: import paths, the ``gpu`` marker, shared fixtures.

``-m "not gpu"`` runs on any machine (oracle against the reference's golden vectors,
host logic, the C-ABI library loads and exports its symbols); ``-m gpu`` are the parity
tests of the CUDA engine and need a B200.
"""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "fwi-edu_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); the CUDA engine's parity tests")


_gpu = None


def gpu_available() -> bool:
    global _gpu
    if _gpu is None:
        try:
            import ctypes
            rt = None
            for name in ("libcudart.so", "libcudart.so.12"):
                try:
                    rt = ctypes.CDLL(name)
                    break
                except OSError:
                    continue
            if rt is None:
                import torch
                _gpu = bool(torch.cuda.is_available())
            else:
                n = ctypes.c_int(0)
                _gpu = rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
        except Exception:
            _gpu = False
    return _gpu


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def port32():
    import pyoracle
    return pyoracle.Port(32)


@pytest.fixture(scope="session")
def port64():
    import pyoracle
    return pyoracle.Port(64)
