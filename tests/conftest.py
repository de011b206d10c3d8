import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the cuda device kernels)")


@pytest.fixture(scope="session")
def oracle():
    """The oracle module (C++ restatement of the reference CPU device)."""
    from oracle import pyoracle
    pyoracle.build(fast=False)
    return pyoracle


@pytest.fixture(scope="session")
def vkl():
    """The cuda device binding; requires a GPU and the built library."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openvkl_b200 import build, vkl as V
    build.build()
    V.load_library()
    return V


@pytest.fixture(scope="session")
def device(vkl):
    return vkl.Device("cuda")


def bits(a):
    """float32 array -> uint32 bit patterns for bit-exact comparison.

    Every NaN maps to one pattern: arithmetic on a NaN background returns the
    canonical NaN on the GPU but keeps the operand's payload on x86, and
    both mean "undefined"; all non-NaN values compare bit for bit."""
    a = np.array(a, np.float32, copy=True)
    a[np.isnan(a)] = np.float32(np.nan)
    return a.view(np.uint32)
