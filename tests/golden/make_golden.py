#!/usr/bin/env python
"""Write the golden fixtures: the oracle's outputs for every case of cases.py.

    python tests/golden/make_golden.py

Each <case>.npz holds nsaved, retcode, nsteps, t (packed save times) and u
(packed saved states) of the oracle run.  The inputs are not stored: the
cases rebuild them from the seeded generators.  Rerun this only when the
oracle's restatement changes on purpose, and commit the fixtures with it.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

import __graft_entry__ as ge  # noqa: E402
from cases import CASES  # noqa: E402


def main(names=None):
    tp, orc = ge.load_package(), ge.load_oracle()
    for name, (build, _tol) in CASES.items():
        if names and name not in names:
            continue
        _device, oracle = build(tp)
        r = oracle(orc)
        np.savez_compressed(HERE / f"{name}.npz", nsaved=r.nsaved, retcode=r.retcode, nsteps=r.nsteps, t=r.t, u=r.u)
        print(f"{name}: {r.nsaved.size} trajectories, {r.t.size} saves", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
