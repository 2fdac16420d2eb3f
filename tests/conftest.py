"""Shared test setup: import paths, the `gpu` marker, common fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "welcome-youtube_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


# the 4x4 repulsion matrix of the workloads (W, H, T, P), embedded in 8x8
def amat_config(a_wt=75.0):
    a = np.full((8, 8), 25.0)

    def s(i, j, v):
        a[i, j] = a[j, i] = v

    s(0, 2, a_wt)
    s(3, 2, 75.0)
    s(1, 2, 50.0)
    s(0, 1, 25.0)
    s(0, 3, 25.0)
    s(1, 3, 25.0)
    return a


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
