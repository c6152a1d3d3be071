"""Shared test setup: import paths for the package and the oracle, and the `gpu` marker.

Tests marked `gpu` need an sm_100 device and call the product through its C ABI; everything
else runs on the CPU (the oracle against the reference's own known answers, host logic, and the
library's exported symbols).
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "n-body_b200"), os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); calls the CUDA library")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def nb():
    import nbody_b200

    nbody_b200.lib()
    return nbody_b200


def rel_err(a, ref):
    """Per-target |a - ref| / |ref| over the first three components."""
    a = np.asarray(a, np.float64)[:, :3]
    ref = np.asarray(ref, np.float64)[:, :3]
    den = np.linalg.norm(ref, axis=1)
    num = np.linalg.norm(a - ref, axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
