"""solve() -- the reference's entry point, routed to the B200 library.

Mirrors TestParticle.solve for
  * TraceProblem with Boris() / MultistepBoris{N}(n)       src/boris/boris.jl:88-114
  * TraceProblem with AdaptiveBoris / AdaptiveMultistep    src/boris/adaptive_boris.jl:21-38
  * TraceGCProblem with alg = :rk4 / :rk45                 src/gc/gc_solver.jl:59-102
with the same keywords and defaults.  prob_func is applied on the host for
every trajectory to build the (6, N) initial-state table, as the reference's
GPU path does (src/boris/boris_kernel.jl:290-294); a (6, N) u0 can be passed
instead.  Only EnsembleB200 runs here: there is no CPU fallback.
"""
from __future__ import annotations

import os
import threading
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi
from .fields import as_field
from .problems import (_ADIA, AdaptiveHybrid, Boris, EnsembleB200, EnsembleContext, MultistepBoris,
                       TraceGCProblem, TraceHybridProblem, TraceProblem, as_term)
from .runtime import Context
from .solution import EnsembleSolution

_PREC = {"fp64": _abi.TP_PREC_FP64, "fp32c": _abi.TP_PREC_FP32C}
_SCHED = {"auto": _abi.TP_SCHED_AUTO, "static": _abi.TP_SCHED_STATIC, "queue": _abi.TP_SCHED_QUEUE}
_GC_PREC = {"fp64": _abi.TP_GC_PREC_FP64, "fp32": _abi.TP_GC_PREC_FP32RHS, "fp32rhs": _abi.TP_GC_PREC_FP32RHS,
            "fp32c": _abi.TP_GC_PREC_FP32RHS}


def _rows_of(table: np.ndarray) -> np.ndarray:
    """(N, width) C-contiguous copy of a (width, N) table: particle-major, the
    library's layout.  Large tables are transposed by several host threads
    (numpy's copy releases the GIL), each in blocks of 32768 particles that
    stay in cache (1e6 x 6: 8.7 -> 3.8 ms on 8 cores)."""
    n = table.shape[1]
    if n < (1 << 18) or table.flags["F_CONTIGUOUS"]:
        return np.ascontiguousarray(table.T)
    out = np.empty((n, table.shape[0]))
    k = max(1, min(8, os.cpu_count() or 1))
    step = (n + k - 1) // k
    blk = 32768

    def part(a):
        end = min(n, a + step)
        for b in range(a, end, blk):
            e = min(b + blk, end)
            np.copyto(out[b:e], table[:, b:e].T)

    threads = [threading.Thread(target=part, args=(a,)) for a in range(0, n, step)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    return out


def _initial_table(prob, trajectories: int, width: int) -> np.ndarray:
    u0 = np.asarray(prob.u0, dtype=np.float64)
    if u0.ndim == 2:
        if u0.shape[0] != width:
            raise ValueError(f"u0 table must be ({width}, N)")
        if prob.prob_func is not None:
            raise ValueError("pass either a (width, N) u0 table or a prob_func, not both")
        if trajectories not in (1, u0.shape[1]):
            raise ValueError("trajectories must equal the number of u0 columns")
        return _rows_of(u0)
    if u0.shape != (width,):
        raise ValueError(f"u0 must have {width} components")
    if prob.prob_func is None:
        return np.tile(u0, (trajectories, 1))
    out = np.empty((trajectories, width))
    for i in range(trajectories):
        new = prob.prob_func(prob, EnsembleContext(i + 1))
        out[i] = np.asarray(new.u0, dtype=np.float64)
    return out


@dataclass
class BorisPlan:
    """Everything a full-orbit solve hands to the library (also used by the tests)."""

    desc: _abi.RunDesc
    E: object
    B: object
    u0: np.ndarray          # (N, 6)
    dt_i: Optional[np.ndarray]
    tend_i: Optional[np.ndarray]
    alg_name: str
    device: int


@dataclass
class GCPlan:
    desc: _abi.GCDesc
    E: object
    B: object
    y0: np.ndarray          # (N, 4)
    q_i: Optional[np.ndarray]
    q2m_i: Optional[np.ndarray]
    mu_i: Optional[np.ndarray]
    dt_i: Optional[np.ndarray]
    tend_i: Optional[np.ndarray]
    alg_name: str
    device: int


def plan_boris(prob, balg, ens=None, *, trajectories=1, savestepinterval=1, dt=None, isoutside=None,
               save_start=True, save_end=True, save_everystep=True, save_fields=False, save_work=False,
               maxiters=None, step_cap=0, tend=None) -> BorisPlan:
    ens = ens if ens is not None else EnsembleB200()
    if not isinstance(ens, EnsembleB200):
        raise NotImplementedError("this package runs ensembles on the B200 only: use EnsembleB200()")
    adaptive = getattr(balg, "adaptive", False)
    if not adaptive and dt is None:
        raise TypeError("solve() with a fixed-step Boris algorithm needs dt")
    q2m, m, E, B, _F = prob.p
    E, B = as_field(E), as_field(B)
    desc = _abi.RunDesc()
    if isinstance(balg, MultistepBoris):
        desc.alg = _abi.TP_ALG_ADAPTIVE_MULTISTEP if adaptive else _abi.TP_ALG_MULTISTEP
        desc.order = balg.N
        desc.nsub = balg.n
    elif isinstance(balg, Boris):
        desc.alg = _abi.TP_ALG_ADAPTIVE if adaptive else _abi.TP_ALG_BORIS
        desc.order, desc.nsub = 2, 1
    else:
        raise TypeError(f"unsupported algorithm {balg!r}")
    desc.safety = float(balg.safety)
    desc.precision = _PREC[ens.precision]
    desc.t0, desc.t1 = float(prob.tspan[0]), float(prob.tspan[1])
    dt_arr = None
    if dt is not None and np.ndim(dt) > 0:
        dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        desc.dt = float(dt_arr[0]) if dt_arr.size else 0.0
    elif dt is not None:
        desc.dt = float(dt)
    desc.q2m, desc.m = float(q2m), float(m)
    desc.savestepinterval = int(savestepinterval)
    desc.maxiters = int(1_000_000 if maxiters is None else maxiters)
    desc.save_start, desc.save_end = int(save_start), int(save_end)
    desc.save_everystep, desc.save_fields = int(save_everystep), int(save_fields)
    desc.save_work = int(save_work)
    desc.term = as_term(isoutside).descriptor()
    desc.step_cap = int(step_cap)
    desc.schedule = _SCHED[ens.schedule]
    desc.block = int(ens.block)
    desc.particles_per_thread = int(ens.particles_per_thread)
    desc.budget_s = float(ens.budget_s)
    u0 = _initial_table(prob, trajectories, 6)
    tend_arr = None if tend is None else np.ascontiguousarray(tend, dtype=np.float64)
    name = {_abi.TP_ALG_BORIS: "boris", _abi.TP_ALG_MULTISTEP: "multistep_boris",
            _abi.TP_ALG_ADAPTIVE: "adaptive_boris",
            _abi.TP_ALG_ADAPTIVE_MULTISTEP: "adaptive_multistep_boris"}[desc.alg]
    return BorisPlan(desc, E, B, u0, dt_arr, tend_arr, name, ens.device)


def plan_gc(prob, ens=None, *, trajectories=1, savestepinterval=1, dt=None, isoutside=None,
            save_start=True, save_end=True, save_everystep=True, alg="rk4", abstol=1.0e-6,
            reltol=1.0e-6, maxiters=10000, save_fields=False, save_work=False, tend=None) -> GCPlan:
    ens = ens if ens is not None else EnsembleB200()
    if not isinstance(ens, EnsembleB200):
        raise NotImplementedError("this package runs ensembles on the B200 only: use EnsembleB200()")
    alg = str(alg).lstrip(":")
    if alg not in ("rk4", "rk45"):
        import warnings
        warnings.warn("Only :rk4 and :rk45 are supported for native TraceGCProblem currently. Using :rk4.")
        alg = "rk4"
    q, q2m, mu, E, B = prob.p[:5]
    desc = _abi.GCDesc()
    desc.alg = _abi.TP_GC_RK4 if alg == "rk4" else _abi.TP_GC_RK45
    desc.precision = _GC_PREC[ens.precision]
    desc.t0, desc.t1 = float(prob.tspan[0]), float(prob.tspan[1])
    desc.dt_given = int(dt is not None)
    dt_arr = None
    if dt is not None and np.ndim(dt) > 0:
        dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        desc.dt = float(dt_arr[0]) if dt_arr.size else 0.0
    else:
        desc.dt = float(dt) if dt is not None else 0.0
    tend_arr = None if tend is None else np.ascontiguousarray(tend, dtype=np.float64)
    pp_mu = pp_q = pp_q2m = None
    if np.ndim(mu) > 0:
        pp_mu = np.ascontiguousarray(mu, dtype=np.float64)
        desc.mu = 0.0
    else:
        desc.mu = float(mu)
    if np.ndim(q) > 0:  # extension: per-particle charge / charge-to-mass arrays
        pp_q = np.ascontiguousarray(q, dtype=np.float64)
        pp_q2m = np.ascontiguousarray(q2m, dtype=np.float64)
        desc.q, desc.q2m = 0.0, 0.0
    else:
        desc.q, desc.q2m = float(q), float(q2m)
    desc.abstol, desc.reltol = float(abstol), float(reltol)
    desc.savestepinterval = int(savestepinterval)
    desc.maxiters = int(maxiters)
    desc.save_start, desc.save_end = int(save_start), int(save_end)
    desc.save_everystep, desc.save_fields = int(save_everystep), int(save_fields)
    desc.save_work = int(save_work)
    desc.term = as_term(isoutside).descriptor()
    desc.block = int(ens.block)
    desc.budget_s = float(ens.budget_s)
    y0 = _initial_table(prob, trajectories, 4)
    return GCPlan(desc, as_field(E), as_field(B), y0, pp_q, pp_q2m, pp_mu, dt_arr, tend_arr, alg, ens.device)


@dataclass
class AdjointPlan:
    desc: _abi.AdjDesc
    E: object
    B: object
    u0: np.ndarray          # (N, 6)
    device: int


def plan_adjoint(prob, ens=None, *, dt, trajectories: int = 1, checkpoint_every: int = 0,
                 maxiters=None) -> AdjointPlan:
    """Descriptor of the discrete adjoint of solve(prob, Boris(); dt) (final save, no saves in between).

    The adjoint runs in the FP32C arithmetic of EnsembleB200(precision="fp32c")
    with static fields and no termination predicate.  checkpoint_every = 0
    lets the library choose the segment length: 2 steps for an interleaved
    E/B grid when the tape (48 bytes per particle per segment) fits in half
    of the free device memory, else 64.
    """
    ens = ens if ens is not None else EnsembleB200(precision="fp32c")
    if ens.precision != "fp32c":
        raise NotImplementedError("the Boris adjoint runs in precision='fp32c'")
    p = plan_boris(prob, Boris(), ens, dt=dt, trajectories=trajectories, savestepinterval=1,
                   save_start=False, save_everystep=False, maxiters=maxiters)
    d = _abi.AdjDesc()
    d.run = p.desc
    d.checkpoint_every = int(checkpoint_every)
    return AdjointPlan(d, p.E, p.B, p.u0, p.device)


def adjoint_solve(prob, ens=None, *, dt, trajectories: int = 1, checkpoint_every: int = 0, maxiters=None):
    """(final states (N, 6), Tape): tape.backward(dL/d final states) gives the gradients."""
    p = plan_adjoint(prob, ens, dt=dt, trajectories=trajectories, checkpoint_every=checkpoint_every,
                     maxiters=maxiters)
    ctx = Context.get(p.device)
    return ctx.adjoint_forward(p.desc, p.E, p.B, p.u0)


@dataclass
class HybridPlan:
    desc: _abi.HybridDesc
    E: object
    B: object
    u0: np.ndarray          # (N, 6)
    device: int


def plan_hybrid(prob, alg, ens=None, *, trajectories=1, savestepinterval=1, isoutside=None, save_start=True,
                save_end=True, save_everystep=True) -> HybridPlan:
    """Descriptor of solve(::TraceHybridProblem, ::AdaptiveHybrid) (src/hybrid.jl:123-138)."""
    ens = ens if ens is not None else EnsembleB200()
    if not isinstance(ens, EnsembleB200):
        raise NotImplementedError("this package runs ensembles on the B200 only: use EnsembleB200()")
    if not isinstance(alg, AdaptiveHybrid):
        raise TypeError("solve(::TraceHybridProblem, ::AdaptiveHybrid)")
    if ens.precision != "fp64":
        raise NotImplementedError("the hybrid solver runs in precision='fp64'")
    q2m, m, E, B, _F = prob.p
    d = _abi.HybridDesc()
    d.t0, d.t1 = float(prob.tspan[0]), float(prob.tspan[1])
    d.q2m, d.m = float(q2m), float(m)
    d.threshold_gc_to_fo, d.threshold_fo_to_gc = alg.threshold_gc_to_fo, alg.threshold_fo_to_gc
    d.dtmin, d.dtmax, d.safety_fo = alg.dtmin, alg.dtmax, alg.safety_fo
    d.abstol, d.reltol = alg.abstol, alg.reltol
    d.maxiters, d.check_interval = alg.maxiters, alg.check_interval
    d.savestepinterval = int(savestepinterval)
    d.adiabaticity = _ADIA[alg.adiabaticity]
    d.save_adiabaticity = int(alg.save_adiabaticity)
    d.save_start, d.save_end, d.save_everystep = int(save_start), int(save_end), int(save_everystep)
    d.block = int(ens.block)
    d.term = as_term(isoutside).descriptor()
    d.budget_s = float(ens.budget_s)
    return HybridPlan(d, as_field(E), as_field(B), _initial_table(prob, trajectories, 6), ens.device)


def solve(prob, *args, trajectories: int = 1, savestepinterval: int = 1, dt=None, isoutside=None,
          save_start: bool = True, save_end: bool = True, save_everystep: bool = True,
          save_fields: bool = False, save_work: bool = False, maxiters=None, alg=None,
          abstol: float = 1.0e-6, reltol: float = 1.0e-6, step_cap: int = 0, tend=None,
          batch_size=None, seed=None) -> EnsembleSolution:
    """TestParticle.solve(prob, alg, ensemblealg=EnsembleB200(); kwargs...)."""
    if isinstance(prob, TraceHybridProblem):
        if not args:
            raise TypeError("solve(prob::TraceHybridProblem, alg::AdaptiveHybrid, [ensemblealg]; kwargs...)")
        p = plan_hybrid(prob, args[0], args[1] if len(args) > 1 else None, trajectories=trajectories,
                        savestepinterval=savestepinterval, isoutside=isoutside, save_start=save_start,
                        save_end=save_end, save_everystep=save_everystep)
        ctx = Context.get(p.device)
        t0 = time.perf_counter()
        r, ra = ctx.hybrid_run(p.desc, p.E, p.B, p.u0, adiabaticity=bool(p.desc.save_adiabaticity))
        wall = time.perf_counter() - t0
        adia = None if ra is None else (ra.nsaved, ra.t, ra.u)
        return EnsembleSolution(r.t, r.u, r.nsaved, r.retcode, r.nsteps, "hybrid", r.elapsed_ms * 1e-3, wall,
                                prob=prob, adiabaticity=adia)
    if isinstance(prob, TraceGCProblem):
        p = plan_gc(prob, args[0] if args else None, trajectories=trajectories,
                    savestepinterval=savestepinterval, dt=dt, isoutside=isoutside, save_start=save_start,
                    save_end=save_end, save_everystep=save_everystep, alg=alg or "rk4", abstol=abstol,
                    reltol=reltol, maxiters=10000 if maxiters is None else maxiters,
                    save_fields=save_fields, save_work=save_work, tend=tend)
        ctx = Context.get(p.device)
        t0 = time.perf_counter()
        r = ctx.gc_run(p.desc, p.E, p.B, p.y0, p.q_i, p.q2m_i, p.mu_i, p.dt_i, p.tend_i)
        wall = time.perf_counter() - t0
        return EnsembleSolution(r.t, r.u, r.nsaved, r.retcode, r.nsteps, p.alg_name, r.elapsed_ms * 1e-3, wall,
                                prob=prob)
    if not isinstance(prob, TraceProblem):
        raise TypeError("prob must be a TraceProblem or TraceGCProblem")
    if not args:
        raise TypeError("solve(prob::TraceProblem, alg, [ensemblealg]; kwargs...)")
    p = plan_boris(prob, args[0], args[1] if len(args) > 1 else None, trajectories=trajectories,
                   savestepinterval=savestepinterval, dt=dt, isoutside=isoutside, save_start=save_start,
                   save_end=save_end, save_everystep=save_everystep, save_fields=save_fields,
                   save_work=save_work, maxiters=maxiters, step_cap=step_cap, tend=tend)
    ctx = Context.get(p.device)
    if getattr(args[1] if len(args) > 1 else None, "autotune", False):
        key = (p.desc.alg, p.desc.precision, id(p.E), id(p.B), p.desc.term.flags != 0)
        if key not in ctx.tuned_keys:
            ctx.autotune(p.desc, p.E, p.B, p.u0)
            ctx.tuned_keys.add(key)
    t0 = time.perf_counter()
    r = ctx.boris_run(p.desc, p.E, p.B, p.u0, p.dt_i, p.tend_i)
    wall = time.perf_counter() - t0
    return EnsembleSolution(r.t, r.u, r.nsaved, r.retcode, r.nsteps, p.alg_name, r.elapsed_ms * 1e-3, wall,
                            prob=prob)


def prepare_gc(xv, E, B, *, species=None, q=None, m=None, t: float = 0.0, device: int = 0):
    """prepare_gc(xv, E, B; species, q, m) -> (stateinit_gc, (q, q2m, mu, E, B)).

    Computed on the device (src/gc/gc.jl:13-84).  Extension: xv may be a
    (6, N) table; the result is then a (4, N) table and an array of mu.
    """
    from .constants import Proton
    from .problems import _species
    qq, mm = _species(species if species is not None else Proton, q, m)
    E, B = as_field(E), as_field(B)
    xv = np.asarray(xv, dtype=np.float64)
    table = xv.ndim == 2
    xs = xv.T if table else xv.reshape(1, 6)
    y0, mu = Context.get(device).gc_prepare(E, B, xs, qq, mm, t)
    if table:
        return y0.T.copy(), (qq, qq / mm, mu, E, B)
    return y0[0], (qq, qq / mm, float(mu[0]), E, B)


def full_to_gc(xu, param, t: float = 0.0, device: int = 0):
    """full_to_gc(xu, param, t) -> (state_gc, mu) (src/gc/gc.jl:86-102), on the device.

    param is the full-orbit parameter tuple of prepare(): (q2m, m, E, B, F).
    Extension: xu may be a (6, N) table; the result is then a (4, N) table
    and an array of mu.
    """
    q2m, m, E, B = param[0], param[1], as_field(param[2]), as_field(param[3])
    xu = np.asarray(xu, dtype=np.float64)
    table = xu.ndim == 2
    xs = xu.T if table else xu.reshape(1, 6)
    y, mu = Context.get(device).gc_prepare(E, B, xs, q2m * m, m, t)
    if table:
        return y.T.copy(), mu
    return y[0], float(mu[0])


def gc_to_full(state_gc, param, mu, phase=0.0, *, t: float = 0.0, device: int = 0) -> np.ndarray:
    """gc_to_full(state_gc, param, mu, phase=0; t=0) -> xu (src/gc/gc.jl:104-154), on the device.

    param is the full-orbit parameter tuple of prepare(): (q2m, m, E, B, F).
    Extension: state_gc may be a (4, N) table with mu (and phase) scalars or
    arrays of N; the result is then a (6, N) table.
    """
    q2m, m, E, B = param[0], param[1], as_field(param[2]), as_field(param[3])
    y = np.asarray(state_gc, dtype=np.float64)
    table = y.ndim == 2
    ys = y.T if table else y.reshape(1, 4)
    xv = Context.get(device).gc_to_full(E, B, ys, mu, q2m * m, m, phase, t)
    return xv.T.copy() if table else xv[0]
