"""Problem, algorithm and ensemble types mirroring the reference API.

TraceProblem / TraceGCProblem       src/types.jl:25-49, src/gc/gc_solver.jl:8-47
Boris / MultistepBoris / Adaptive*  src/types.jl:51-107
prepare                             src/prepare.jl:93-170
EnsembleB200                        the ensemble algorithm that routes a solve to
                                    the B200 library (the reference dispatches on
                                    the ensemble-algorithm type, boris.jl:137-318)
Terminate*                          flag predicates standing in for `isoutside`
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Any, Callable, Optional

import numpy as np

from . import _abi
from .constants import Proton, Species
from .fields import AbstractField, ZeroField, as_field, build_interpolator, FillExtrap


# ---------------------------------------------------------------- algorithms
@dataclass(frozen=True)
class Boris:
    """Boris() -- fixed-step Boris pusher (Boris{false})."""

    safety: float = 0.0
    adaptive: bool = False


@dataclass(frozen=True)
class MultistepBoris:
    """MultistepBoris{N}(; n=1) -- gyrophase-corrected multistep Boris."""

    N: int = 2
    n: int = 1
    safety: float = 0.0
    adaptive: bool = False

    def __post_init__(self):
        if self.N not in (2, 4, 6):
            raise ValueError("Multistep Boris order N must be 2, 4, or 6.")
        if self.n < 1:
            raise ValueError("Multistep Boris subcycles n must be >= 1")


def MultistepBoris2(n: int = 1) -> MultistepBoris:
    return MultistepBoris(2, n)


def MultistepBoris4(n: int = 1) -> MultistepBoris:
    return MultistepBoris(4, n)


def MultistepBoris6(n: int = 1) -> MultistepBoris:
    return MultistepBoris(6, n)


def AdaptiveBoris(safety: float = 0.1) -> Boris:
    """AdaptiveBoris(; safety) -- dt = safety * 2pi / |q B / m| (src/types.jl:229-237)."""
    return Boris(float(safety), True)


def AdaptiveMultistepBoris(N: int, n: int = 1, safety: float = 0.1) -> MultistepBoris:
    return MultistepBoris(N, n, float(safety), True)


# ---------------------------------------------------------------- ensembles
@dataclass(frozen=True)
class EnsembleB200:
    """Run every trajectory of a solve on one B200.

    precision: "fp64" (the drop-in path, reference operation order) or
               "fp32c" (float32 push with compensated positions).
    schedule:  "auto", "static" (one thread per particle) or "queue"
               (persistent kernel pulling particles from a work queue).
    block:     threads per block (0: library default / tuned).
    particles_per_thread:
               fixed-step solves in analytic fields: 1 or 2 particles advanced
               in lock step by each thread (0: library default / tuned).
    autotune:  time the candidate launch shapes on a sample before the
               first full-orbit solve of each kernel variant (tp_autotune);
               later solves with block = 0, schedule = "auto" and
               particles_per_thread = 0 use the fastest.
    """

    device: int = 0
    precision: str = "fp64"
    schedule: str = "auto"
    block: int = 0
    budget_s: float = 0.0
    autotune: bool = False
    particles_per_thread: int = 0


class EnsembleSerial:  # pragma: no cover - guidance only
    def __init__(self, *a, **k):
        raise NotImplementedError("this package runs ensembles on the B200 only: use EnsembleB200()")


EnsembleThreads = EnsembleSerial


# ---------------------------------------------------------------- termination
@dataclass(frozen=True)
class Terminate:
    """Union of flag predicates replacing the reference's `isoutside` closure."""

    flags: int = 0
    rmin: float = -np.inf
    rmax: float = np.inf
    lo: tuple = (-np.inf, -np.inf, -np.inf)
    hi: tuple = (np.inf, np.inf, np.inf)
    tmax: float = np.inf

    def __or__(self, other: "Terminate") -> "Terminate":
        return Terminate(
            self.flags | other.flags,
            other.rmin if other.flags & _abi.TP_TERM_SHELL else self.rmin,
            other.rmax if other.flags & _abi.TP_TERM_SHELL else self.rmax,
            other.lo if other.flags & _abi.TP_TERM_BOX else self.lo,
            other.hi if other.flags & _abi.TP_TERM_BOX else self.hi,
            other.tmax if other.flags & _abi.TP_TERM_TIME else self.tmax,
        )

    def descriptor(self) -> _abi.TermDesc:
        d = _abi.TermDesc()
        d.flags = self.flags
        d.rmin = float(self.rmin)
        d.rmax = float(self.rmax)
        for k in range(3):
            d.lo[k] = float(self.lo[k])
            d.hi[k] = float(self.hi[k])
        d.tmax = float(self.tmax)
        return d


def TerminateShell(rmin: float = -np.inf, rmax: float = np.inf) -> Terminate:
    """Outside when |x| < rmin or |x| > rmax."""
    return Terminate(flags=_abi.TP_TERM_SHELL, rmin=rmin, rmax=rmax)


def TerminateBox(lo=(-np.inf,) * 3, hi=(np.inf,) * 3) -> Terminate:
    """Outside when any x_c < lo_c or x_c > hi_c."""
    return Terminate(flags=_abi.TP_TERM_BOX, lo=tuple(lo), hi=tuple(hi))


def TerminateNaN() -> Terminate:
    """Outside when any state component is NaN."""
    return Terminate(flags=_abi.TP_TERM_NAN)


def TerminateTime(tmax: float) -> Terminate:
    """Outside when t > tmax."""
    return Terminate(flags=_abi.TP_TERM_TIME, tmax=tmax)


def as_term(isoutside) -> Terminate:
    if isoutside is None:
        return Terminate()
    if isinstance(isoutside, Terminate):
        return isoutside
    raise NotImplementedError(
        "isoutside must be a Terminate* predicate (TerminateShell, TerminateBox, TerminateNaN, "
        "TerminateTime, combined with |): callables cannot run on the device")


# ---------------------------------------------------------------- problems
@dataclass
class EnsembleContext:
    """What prob_func receives (SciMLBase.EnsembleContext; sim_id is 1-based)."""

    sim_id: int
    repeat: int = 1


@dataclass
class TraceProblem:
    """TraceProblem(u0, tspan, p; prob_func) -- p = (q2m, m, E, B, F) from prepare().

    Extension: u0 may be a (6, N) table, one column per trajectory.
    """

    u0: Any
    tspan: tuple
    p: tuple
    prob_func: Optional[Callable] = None

    def remake(self, **kw) -> "TraceProblem":
        return replace(self, **kw)


@dataclass
class TraceGCProblem:
    """TraceGCProblem(u0, tspan, p; prob_func) -- p = (q, q2m, mu, E, B) from prepare_gc()."""

    u0: Any
    tspan: tuple
    p: tuple
    prob_func: Optional[Callable] = None

    def remake(self, **kw) -> "TraceGCProblem":
        return replace(self, **kw)


@dataclass
class TraceHybridProblem:
    """TraceHybridProblem(u0, tspan, p; prob_func) -- full-orbit u0 (6 values, or a
    (6, N) table) and p = (q2m, m, E, B, F) (src/hybrid.jl:85-120)."""

    u0: Any
    tspan: tuple
    p: tuple
    prob_func: Optional[Callable] = None

    def remake(self, **kw) -> "TraceHybridProblem":
        return replace(self, **kw)


_ADIA = {"curvature": 0, "gradB": 1, "both": 2, "jacobian": 3}


@dataclass(frozen=True)
class AdaptiveHybrid:
    """AdaptiveHybrid(; threshold, threshold_gc_to_fo, threshold_fo_to_gc, dtmax, dtmin,
    safety_fo, abstol, reltol, maxiters, check_interval, adiabaticity, save_adiabaticity)
    (src/hybrid.jl:41-83): GC (RK45) while adiabatic, Boris full orbit otherwise."""

    threshold_gc_to_fo: float
    threshold_fo_to_gc: float
    dtmin: float
    dtmax: float
    safety_fo: float = 0.1
    abstol: float = 1.0e-6
    reltol: float = 1.0e-6
    maxiters: int = 10000
    check_interval: int = 10
    adiabaticity: str = "curvature"
    save_adiabaticity: bool = True

    def __init__(self, *, threshold: float = 0.1, threshold_gc_to_fo=None, threshold_fo_to_gc=None, dtmax,
                 dtmin=None, safety_fo: float = 0.1, abstol: float = 1.0e-6, reltol: float = 1.0e-6,
                 maxiters: int = 10000, check_interval: int = 10, adiabaticity="curvature",
                 save_adiabaticity: bool = True):
        gc_fo = threshold if threshold_gc_to_fo is None else threshold_gc_to_fo
        fo_gc = threshold if threshold_fo_to_gc is None else threshold_fo_to_gc
        adia = str(adiabaticity).lstrip(":")
        if check_interval <= 0:
            raise ValueError("check_interval must be positive.")
        if not gc_fo >= fo_gc:
            raise ValueError("threshold_gc_to_fo must be >= threshold_fo_to_gc for hysteresis.")
        if adia not in _ADIA:
            raise ValueError("adiabaticity must be one of :curvature, :gradB, :both, :jacobian.")
        for k, v in dict(threshold_gc_to_fo=float(gc_fo), threshold_fo_to_gc=float(fo_gc),
                         dtmin=float(1.0e-2 * dtmax if dtmin is None else dtmin), dtmax=float(dtmax),
                         safety_fo=float(safety_fo), abstol=float(abstol), reltol=float(reltol),
                         maxiters=int(maxiters), check_interval=int(check_interval), adiabaticity=adia,
                         save_adiabaticity=bool(save_adiabaticity)).items():
            object.__setattr__(self, k, v)


def remake(prob, **kw):
    return prob.remake(**kw)


def _species(species, q, m):
    if isinstance(species, str):
        from .constants import SpeciesDict
        species = SpeciesDict[species]
    q = species.q if q is None else q
    m = species.m if m is None else m
    return float(q), float(m)


def prepare(*args, species: Species = Proton, q=None, m=None, order: int = 1, bc=None,
            E=None, F=None, gridtype=None, **kw):
    """prepare(E, B, F=ZeroField(); species, q, m) -> (q2m, m, E, B, F).

    Also prepare(x, y, z, E, B, F; order, bc, gridtype) with E, B given as
    (3, n1, n2, n3) arrays on the grid axes (gridtype CartesianGrid,
    RectilinearGrid or StructuredGrid), and prepare(B; E=ZeroField())
    (src/prepare.jl:136-170).
    """
    qq, mm = _species(species, q, m)
    if len(args) >= 5:
        x, y, z, Ea, Ba = args[:5]
        Fa = args[5] if len(args) > 5 else ZeroField()
        bc = bc if bc is not None else FillExtrap()

        def grid(a):
            if isinstance(a, np.ndarray) and a.ndim == 4:
                if gridtype is None:
                    return build_interpolator(a, x, y, z, order, bc)
                return build_interpolator(gridtype, a, x, y, z, order, bc)
            return as_field(a)

        return (qq / mm, mm, grid(Ea), grid(Ba), as_field(Fa))
    if len(args) == 1:
        return (qq / mm, mm, as_field(E if E is not None else ZeroField()), as_field(args[0]),
                as_field(F if F is not None else ZeroField()))
    if len(args) in (2, 3):
        Fa = args[2] if len(args) == 3 else (F if F is not None else ZeroField())
        return (qq / mm, mm, as_field(args[0]), as_field(args[1]), as_field(Fa))
    raise TypeError("prepare(E, B[, F]), prepare(B; E=...) or prepare(x, y, z, E, B[, F])")
