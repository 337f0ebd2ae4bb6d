"""Test configuration: import paths, the `gpu` marker, shared fixtures.

`-m "not gpu"` tests run on CPU only (oracle vs golden vectors, host logic,
the C ABI library loading and exporting its symbols).  `-m gpu` tests call the
CUDA kernels through the C ABI and compare with the oracle.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rips2026-amd_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# a solve that has not finished in 10 s has gone wrong: fail it on the device
# (bounded waits return B2_TIMEOUT) instead of waiting out the 20 s default
os.environ.setdefault("B2_TIMEOUT_MS", "10000")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return load


@pytest.fixture(scope="session")
def b2():
    import b200sssp
    return b200sssp


@pytest.fixture(scope="session")
def orc():
    import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch
