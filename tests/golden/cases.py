"""The golden cases: small seeded runs of the benchmark configurations.

Each case builds its inputs from the seeded generators of
testparticle_b200.workloads (SplitMix64 streams: identical tables on every
machine), so a fixture stores only the outputs.  `make_golden.py` writes the
oracle's outputs to <name>.npz; `tests/test_golden.py` checks that the oracle
still reproduces them bit for bit (CPU) and that the device path matches them
within the case's bar (GPU).

A case is (build, tol): build(tp) returns (device, oracle), two callables
that run the same problem through solve() and through the oracle; tol is the
bar on the saved states and times of the device run (1e-13 where the
arithmetic is +, -, *, /, sqrt on both sides; 1e-10 where CUDA's and glibc's
atan / sincos / pow may differ in the last bit).
"""
from __future__ import annotations

import math

import numpy as np


def _boris(tp, prob, alg, prec="fp64", **kw):
    def device():
        return tp.solve(prob, alg, tp.EnsembleB200(precision=prec), **kw)

    def oracle(orc):
        p = tp.plan_boris(prob, alg, tp.EnsembleB200(precision="fp64"), **kw)
        return orc.boris_run(p.desc, p.E, p.B, p.u0, p.dt_i, p.tend_i)

    return device, oracle


def config1_boris(tp):
    w = tp.workloads.config1(64)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    return _boris(tp, prob, tp.Boris(), dt=w.dt, savestepinterval=w.savestepinterval)


def _grid_workload(tp):
    w = tp.workloads.config2(n=128, nx=32, nt=500, ssi=100)
    return w, tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))


def config2_boris_grid(tp):
    w, prob = _grid_workload(tp)
    return _boris(tp, prob, tp.Boris(), dt=w.dt, savestepinterval=w.savestepinterval, save_fields=True)


def config2_cubic_grid(tp):
    w, _ = _grid_workload(tp)
    dx = 1.0e5
    g = np.arange(32) * dx
    Ea, Ba, _L = tp.workloads.turbulent_grid(32, dx, 5.0e-9)
    E = tp.build_interpolator(Ea, g, g, g, 3, tp.PeriodicBC("exclusive"))
    B = tp.build_interpolator(Ba, g, g, g, 3, tp.PeriodicBC("exclusive"))
    prob = tp.TraceProblem(w.u0[:, :64].copy(), (0.0, 300 * w.dt), tp.prepare(E, B, species=w.species))
    return _boris(tp, prob, tp.Boris(), dt=w.dt, savestepinterval=50)


def _regular_dipole(tp, n=64, nt=2000, ssi=200):
    w = tp.workloads.config3(4 * n, nt=nt, ssi=ssi)
    keep = np.flatnonzero(w.extra["Ek_eV"] < 1.0e6)[:n]
    prob = tp.TraceProblem(w.u0[:, keep].copy(), w.tspan, tp.prepare(w.E, w.B, species=tp.Proton))
    return w, keep, prob


def config3_adaptive(tp):
    w, keep, prob = _regular_dipole(tp)
    return _boris(tp, prob, tp.AdaptiveBoris(0.1), tend=w.tend[keep], savestepinterval=w.savestepinterval,
                  isoutside=w.isoutside, step_cap=2000)


def config3_multistep(tp):
    w, keep, prob = _regular_dipole(tp)
    return _boris(tp, prob, tp.MultistepBoris4(2), dt=w.dt[keep], tend=w.tend[keep],
                  savestepinterval=w.savestepinterval, isoutside=w.isoutside)


def _gc(tp, alg):
    w = tp.workloads.config4(64)
    prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
    kw = dict(tend=w.tau_b, alg=alg, savestepinterval=20, maxiters=100_000)
    kw.update(dict(dt=w.tau_b / 200) if alg == "rk4" else dict(abstol=1e-9, reltol=1e-6))

    def device():
        return tp.solve(prob, tp.EnsembleB200(precision="fp64"), **kw)

    def oracle(orc):
        p = tp.plan_gc(prob, **kw)
        return orc.gc_run(p.desc, p.E, p.B, p.y0, p.q_i, p.q2m_i, p.mu_i, dt_i=p.dt_i, tend_i=p.tend_i)

    return device, oracle


def config4_gc_rk4(tp):
    return _gc(tp, "rk4")


def config4_gc_rk45(tp):
    return _gc(tp, "rk45")


def hybrid_bottle(tp):
    B0, alpha = 1.0e-4, 1.0e-2
    T = 2 * math.pi / (abs(tp.qi / tp.mi) * B0)
    rng = tp.workloads.SplitMix64(tp.workloads.SEED0 + 61)
    n = 32
    u0 = np.zeros((6, n))
    u0[:3] = rng.normal(3 * n, 0.5).reshape(3, n)
    vperp = rng.uniform(n, 2.0e4, 8.0e4)
    ph = rng.uniform(n, 0.0, 2 * math.pi)
    u0[3], u0[4] = vperp * np.cos(ph), vperp * np.sin(ph)
    u0[5] = rng.uniform(n, -1.2e5, 1.2e5)
    prob = tp.TraceHybridProblem(u0, (0.0, 10 * T), tp.prepare(tp.ZeroField(), tp.QuadraticField.bottle(B0, alpha),
                                                               species=tp.Proton))
    alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=T, dtmin=1.0e-4 * T, check_interval=100, save_adiabaticity=False)

    def device():
        return tp.solve(prob, alg, savestepinterval=5)

    def oracle(orc):
        p = tp.plan_hybrid(prob, alg, savestepinterval=5)
        r, _ = orc.hybrid_run(p.desc, p.E, p.B, p.u0)
        return r

    return device, oracle


CASES = {
    "config1_boris": (config1_boris, 1e-13),
    "config2_boris_grid": (config2_boris_grid, 1e-13),
    "config2_cubic_grid": (config2_cubic_grid, 1e-13),
    "config3_adaptive": (config3_adaptive, 1e-13),
    "config3_multistep": (config3_multistep, 1e-10),
    "config4_gc_rk4": (config4_gc_rk4, 1e-13),
    "config4_gc_rk45": (config4_gc_rk45, 1e-10),
    "hybrid_bottle": (hybrid_bottle, 1e-13),
}
