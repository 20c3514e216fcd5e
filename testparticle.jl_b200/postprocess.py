"""get_fields / get_work on solutions, evaluated on the device.

The reference's post-processing (src/boris/boris.jl:594-640): the fields at
every saved state, and the work rates of get_work_rates
(src/equations.jl:394-441) or get_work_rates_gc (:445-480).  Both run through
tp_eval_points, the kernel that also fills the saved columns of save_fields /
save_work, so the results equal those columns.
"""
from __future__ import annotations

import numpy as np

from .fields import as_field
from .problems import TraceGCProblem
from .runtime import Context
from .solution import EnsembleSolution, TraceSolution


def _states(sol):
    if isinstance(sol, (TraceSolution, EnsembleSolution)):
        if sol.prob is None:
            raise ValueError("the solution does not carry its problem (solve it with this package's solve)")
        if isinstance(sol, TraceSolution):
            return sol.prob, np.asarray(sol.u), np.asarray(sol.t), [sol.index] * len(sol.t)
        idx = np.repeat(np.arange(sol.nsaved.size), sol.nsaved)
        return sol.prob, np.asarray(sol.u_all), np.asarray(sol.t_all), idx
    raise TypeError("get_fields / get_work take a TraceSolution or an EnsembleSolution")


def _eval(sol, want: int, device: int = 0):
    prob, u, t, idx = _states(sol)
    ctx = Context.get(device)
    if isinstance(prob, TraceGCProblem):
        q, q2m, mu, E, B = prob.p[:5]
        E, B = as_field(E), as_field(B)
        # per-particle q, q2m, mu (an extension) become one value per saved
        # state, so the whole ensemble is still one launch
        idx = np.asarray(idx)
        per_state = (lambda a: np.asarray(a, dtype=np.float64).reshape(-1)[idx]  # noqa: E731
                     if np.ndim(a) > 0 else float(a))
        return ctx.eval_points(E, B, u, t, gc=True, want=want, q2m=per_state(q2m), q=per_state(q),
                               mu=per_state(mu))
    q2m, m, E, B = prob.p[:4]
    return ctx.eval_points(as_field(E), as_field(B), u, t, gc=False, want=want, q2m=q2m, m=m)


def get_fields(sol, device: int = 0):
    """(E, B): the fields at every saved state, each (n_saves, 3)."""
    out = _eval(sol, 1, device)
    return out[:, 0:3], out[:, 3:6]


def get_work(sol, device: int = 0):
    """(n_saves, 4): (P_par, P_fermi, P_grad, P_betatron) at every saved state."""
    return _eval(sol, 2, device)
