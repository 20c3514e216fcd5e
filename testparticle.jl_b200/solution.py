"""Solution containers with the reference's layout.

TraceSolution mirrors the ODESolution that _boris_single builds
(src/boris/boris.jl:553-556): `t` (save times), `u` (one state row per save,
width 6 / 12 with fields), `retcode`, `alg`, and linear interpolation
`sol(t)` (SciMLBase LinearInterpolation).  EnsembleSolution mirrors
SciMLBase.EnsembleSolution: `u[i]` is trajectory i, `elapsedTime` the solve
time.  Trajectories are views into one packed buffer, so a 10^6-particle
solve builds no per-trajectory objects until they are indexed.
"""
from __future__ import annotations

from collections.abc import Sequence

import numpy as np

from . import _abi

RETCODE_NAMES = {
    _abi.TP_RET_DEFAULT: "Default",
    _abi.TP_RET_SUCCESS: "Success",
    _abi.TP_RET_TERMINATED: "Terminated",
    _abi.TP_RET_MAXITERS: "MaxIters",
}


class TraceSolution:
    __slots__ = ("t", "u", "retcode", "alg", "nsteps", "prob", "index", "stats")

    def __init__(self, t: np.ndarray, u: np.ndarray, retcode: str, alg: str, nsteps: int = 0, prob=None,
                 index: int = 0, stats=None):
        self.t = t
        self.u = u
        self.retcode = retcode
        self.alg = alg
        self.nsteps = nsteps
        self.prob = prob      # the problem solved (get_fields / get_work read its fields)
        self.index = index    # trajectory index within its ensemble
        self.stats = stats    # hybrid solves: {"adiabaticity": {"t", "components", "mode"}}

    def __len__(self):
        return self.t.size

    def __getitem__(self, idx):
        """sol[c, k] = component c of save k (Julia's sol[i, j], 0-based here)."""
        if isinstance(idx, tuple):
            c, k = idx
            return self.u[k, c]
        return self.u[idx]

    def __call__(self, t: float) -> np.ndarray:
        """Linear interpolation between saves (SciMLBase LinearInterpolation)."""
        ts = self.t
        if ts.size == 0:
            raise ValueError("empty solution")
        if t <= ts[0]:
            return self.u[0].copy()
        if t >= ts[-1]:
            return self.u[-1].copy()
        i = int(np.searchsorted(ts, t, side="right")) - 1
        th = (t - ts[i]) / (ts[i + 1] - ts[i])
        return (1 - th) * self.u[i] + th * self.u[i + 1]

    def __repr__(self):
        return f"TraceSolution(alg={self.alg}, retcode={self.retcode}, saves={self.t.size})"


class _Trajectories(Sequence):
    def __init__(self, ens: "EnsembleSolution"):
        self._e = ens

    def __len__(self):
        return self._e.nsaved.size

    def __getitem__(self, i):
        e = self._e
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        a, b = e.offsets[i], e.offsets[i + 1]
        stats = None
        if e.adiabaticity is not None:
            na, ta, va = e.adiabaticity
            c, d = e._aoff[i], e._aoff[i + 1]
            stats = {"adiabaticity": {"t": ta[c:d], "components": va[c:d, 0],
                                      "mode": ["GC" if m == 0 else "FO" for m in va[c:d, 1]]}}
        return TraceSolution(e.t_all[a:b], e.u_all[a:b], RETCODE_NAMES.get(int(e.retcodes[i]), "Default"),
                             e.alg, int(e.nsteps[i]), e.prob, i, stats)


class EnsembleSolution:
    """Ensemble of trajectories over packed buffers (t_all, u_all, offsets)."""

    def __init__(self, t_all, u_all, nsaved, retcodes, nsteps, alg: str, elapsed_s: float,
                 elapsed_e2e_s: float = 0.0, prob=None, adiabaticity=None):
        self.prob = prob
        # hybrid solves: (checks per trajectory, check times, (value, mode) rows)
        self.adiabaticity = adiabaticity
        if adiabaticity is not None:
            self._aoff = np.zeros(adiabaticity[0].size + 1, dtype=np.int64)
            np.cumsum(adiabaticity[0], out=self._aoff[1:])
        self.t_all = t_all
        self.u_all = u_all
        self.nsaved = nsaved
        self.retcodes = retcodes
        self.nsteps = nsteps
        self.alg = alg
        self.elapsedTime = elapsed_s
        self.elapsed_e2e = elapsed_e2e_s
        self._offsets = None
        self.u = _Trajectories(self)

    @property
    def offsets(self) -> np.ndarray:
        """Row of each trajectory's first save in t_all / u_all (n + 1 values),
        computed on first use."""
        if self._offsets is None:
            off = np.zeros(self.nsaved.size + 1, dtype=np.int64)
            np.cumsum(self.nsaved, out=off[1:])
            self._offsets = off
        return self._offsets

    def __len__(self):
        return self.nsaved.size

    def __iter__(self):
        return iter(self.u)

    def __getitem__(self, i):
        return self.u[i]

    @property
    def converged(self):
        return True

    def final_states(self) -> np.ndarray:
        """(N, width) array of every trajectory's last saved state (NaN if none)."""
        out = np.full((self.nsaved.size, self.u_all.shape[1]), np.nan)
        has = self.nsaved > 0
        out[has] = self.u_all[self.offsets[1:][has] - 1]
        return out

    def particle_steps(self) -> int:
        return int(self.nsteps.sum())
