"""Shared test set-up: markers, import paths and small systems.

The CPU oracle (oracle/) is the oracle of every parity test; it is imported
only here and in the tests."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libospreydpd_cuda.so")
    config.addinivalue_line("markers", "slow: longer statistical runs")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    import dpd_oracle
    dpd_oracle.build()
    return dpd_oracle


@pytest.fixture(scope="session")
def engine_mod():
    """The CUDA engine; a GPU test fails (not skips) if it cannot load."""
    from osprey_dpd_b200 import build, engine
    build.build()
    engine.load()
    return engine


def rel_err(a, b, scale=None):
    """max |a-b| over beads divided by the RMS magnitude of b."""
    a = np.asarray(a)
    b = np.asarray(b)
    if scale is None:
        scale = float(np.sqrt(np.mean(np.sum(b * b, axis=-1)))) or 1.0
    return float(np.max(np.abs(a - b))) / scale
