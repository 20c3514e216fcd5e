"""Golden fixtures (tests/golden/): the oracle's outputs on seeded inputs.

CPU: the oracle reproduces every fixture bit for bit, so a change to the
restatement that moves any result is caught here.  GPU: the device path
(solve() through the C ABI) matches every fixture: identical save counts,
return codes and step counts, and saved times and states within the case's
bar (tests/golden/cases.py).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

from cases import CASES  # noqa: E402

NAMES = sorted(CASES)


def _fixture(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _rel_rows(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.ndim == 1:
        a, b = a[:, None], b[:, None]
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b))
    a, b = np.where(np.isnan(a), 0.0, a), np.where(np.isnan(b), 0.0, b)
    worst = 0.0
    for lo in range(0, a.shape[1], 3):
        hi = min(lo + 3, a.shape[1])
        d = np.linalg.norm(a[:, lo:hi] - b[:, lo:hi], axis=1)
        r = np.linalg.norm(b[:, lo:hi], axis=1)
        worst = max(worst, float(np.max(d / np.where(r > 0, r, 1.0)))) if d.size else worst
    return worst


def test_fixtures_present():
    for name in NAMES:
        f = _fixture(name)
        assert f["nsaved"].sum() == f["t"].size == f["u"].shape[0] > 0


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(tp, orc, name):
    build, _tol = CASES[name]
    _device, oracle = build(tp)
    r = oracle(orc)
    f = _fixture(name)
    assert np.array_equal(r.nsaved, f["nsaved"])
    assert np.array_equal(r.retcode, f["retcode"])
    assert np.array_equal(r.nsteps, f["nsteps"])
    assert np.array_equal(r.t, f["t"], equal_nan=True)
    assert np.array_equal(r.u, f["u"], equal_nan=True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_matches_fixture(tp, name):
    build, tol = CASES[name]
    device, _oracle = build(tp)
    s = device()
    f = _fixture(name)
    assert np.array_equal(s.nsaved, f["nsaved"])
    assert np.array_equal(s.retcodes, f["retcode"])
    assert np.array_equal(s.nsteps, f["nsteps"])
    assert _rel_rows(s.t_all, f["t"]) <= tol
    assert _rel_rows(s.u_all, f["u"]) <= tol
