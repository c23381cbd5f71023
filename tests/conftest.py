"""Shared test configuration.

Tests marked `gpu` need a B200 and run the CUDA path through the C-ABI; everything else
runs on the CPU (oracle known-answer tests, host logic, library export checks, gloo
multi-process harness).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and the built libjfli_b200.so")


@pytest.fixture(scope="session")
def cosmo():
    from jfli_b200 import Planck18

    return Planck18()


def rel_l2(a, b):
    """||a - b|| / ||b|| over all elements (complex-aware)."""
    a = np.asarray(a)
    b = np.asarray(b)
    dt = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a = a.astype(dt)
    b = b.astype(dt)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
