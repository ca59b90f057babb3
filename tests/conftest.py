"""Test configuration: markers and import paths.

CPU tests (-m "not gpu") cover the oracle against the reference's own kernels
and the golden fixtures, the host set-up code, and the C ABI's library
(symbols, admission checks).  GPU tests (-m gpu) are the parity tests proper
and call the CUDA path through the C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "dm-heom_b200", os.path.join("tests", "golden")):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA path)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_small.npz"))


@pytest.fixture(scope="session")
def root():
    return ROOT
