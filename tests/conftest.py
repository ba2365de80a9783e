"""Shared fixtures: golden vectors, the CPU oracle, the built library.

Markers: ``gpu`` tests need a CUDA device and call libbh_b200 through its C
ABI; everything else runs on the CPU (oracle pins, host logic, ABI layout).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libbh_b200.so")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.build()
    return o


@pytest.fixture(scope="session")
def bhlib():
    """The built C-ABI library (built here with nvcc if missing)."""
    from blackhorizon_b200 import _lib, build

    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    from blackhorizon_b200 import _lib

    _lib.load()
    return torch.device("cuda", 0)
