"""Test configuration: paths, the ``gpu`` marker and shared fixtures.

CPU tests (``-m "not gpu"``) check the oracle against the golden vectors
generated from the reference, the host-side logic and the C-ABI library's
exports.  GPU tests (``-m gpu``) call the CUDA path through the C-ABI and
compare it with the oracle.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
PKG_ROOT = REPO / "blackhole-sim_b200"
for p in (str(REPO), str(PKG_ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def micro_golden():
    return np.load(GOLDEN / "micro_kernels.npz")


@pytest.fixture(scope="session")
def kerr_golden():
    return np.load(GOLDEN / "kerr.npz")


@pytest.fixture(scope="session")
def ray_golden():
    return np.load(GOLDEN / "ray_loop.npz")


def rel_l1(a, b) -> float:
    """rel L1 = sum|a - b| / sum|b| (external_validation.py:110-145)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sum(np.abs(a - b)) / (np.sum(np.abs(b)) + 1e-300))
