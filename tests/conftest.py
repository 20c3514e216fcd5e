"""Shared fixtures.  `gpu` marks tests that need a B200 (run with -m gpu)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def tp():
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    return ge.load_oracle()


def julia_isapprox(a, b, rtol=None, atol=0.0):
    """Julia's isapprox for arrays: norm(a - b) <= max(atol, rtol * max(norm(a), norm(b)))."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    if rtol is None:
        rtol = 0.0 if atol > 0 else np.sqrt(np.finfo(float).eps)
    d = np.linalg.norm(a - b)
    return d <= max(atol, rtol * max(np.linalg.norm(a), np.linalg.norm(b)))
