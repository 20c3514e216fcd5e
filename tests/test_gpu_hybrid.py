"""GPU parity of the adaptive hybrid GC / full-orbit solver (tp_hybrid_run)
against the CPU oracle (src/hybrid.jl:234-474 restated).

Bars: everything on the path uses +, -, *, /, sqrt and fma -- the gyrophase
trigonometry is the portable sin / cos / atan2 of the kernel and the oracle,
because the hybrid's accept / reject and mode decisions turn last-bit
differences into different step sequences (a 1-ulp change of the initial
state changes step counts).  Step counts, check counts and modes are compared
exactly, states and times at 1e-13 relative.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_rows(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b))
    a, b = np.where(np.isnan(a), 0.0, a), np.where(np.isnan(b), 0.0, b)
    d = np.linalg.norm(a - b, axis=-1)
    r = np.linalg.norm(b, axis=-1)
    return float(np.max(d / np.where(r > 0, r, 1.0))) if d.size else 0.0


def _both(tp, orc, prob, alg, **kw):
    sols = tp.solve(prob, alg, **kw)
    plan = tp.plan_hybrid(prob, alg, **kw)
    r, a = orc.hybrid_run(plan.desc, plan.E, plan.B, plan.u0)
    return sols, r, a


def _check(sols, r, a, tol=1e-13):
    assert np.array_equal(sols.nsaved, r.nsaved)
    assert np.array_equal(sols.retcodes, r.retcode)
    assert np.array_equal(sols.nsteps, r.nsteps)
    assert _rel_rows(sols.t_all[:, None], r.t[:, None]) <= tol
    assert _rel_rows(sols.u_all[:, :3], r.u[:, :3]) <= tol
    assert _rel_rows(sols.u_all[:, 3:6], r.u[:, 3:6]) <= tol
    if a is not None:
        na, ta, va = sols.adiabaticity
        assert np.array_equal(na, a.nsaved)
        assert np.array_equal(va[:, 1], a.u[:, 1])          # the mode of every check
        assert _rel_rows(va[:, :1], a.u[:, :1]) <= tol


def _bottle(tp, n=256, seed=3):
    B0, alpha = 1.0e-4, 1.0e-2
    q2m = tp.qi / tp.mi
    T = 2 * math.pi / (abs(q2m) * B0)
    rng = np.random.default_rng(seed)
    u0 = np.zeros((6, n))
    u0[:3] = rng.normal(0.0, 0.5, (3, n))
    vperp = rng.uniform(2.0e4, 8.0e4, n)
    ph = rng.uniform(0, 2 * math.pi, n)
    u0[3], u0[4] = vperp * np.cos(ph), vperp * np.sin(ph)
    u0[5] = rng.uniform(-1.2e5, 1.2e5, n)
    B = tp.QuadraticField.bottle(B0, alpha)
    prob = tp.TraceHybridProblem(u0, (0.0, 30 * T), tp.prepare(tp.ZeroField(), B, species=tp.Proton))
    return prob, T


@pytest.mark.parametrize("mode", ["curvature", "gradB", "both", "jacobian"])
def test_hybrid_bottle_matches_oracle(tp, orc, mode):
    prob, T = _bottle(tp)
    alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=T, dtmin=1.0e-4 * T, check_interval=100, adiabaticity=mode)
    sols, r, a = _both(tp, orc, prob, alg, savestepinterval=5)
    _check(sols, r, a)
    modes = set(sols.adiabaticity[2][:, 1])
    assert modes == {0.0, 1.0}
    assert all(s.retcode == "Success" for s in sols)


def test_hybrid_buffer_band_and_flags(tp, orc):
    prob, T = _bottle(tp, n=128, seed=5)
    alg = tp.AdaptiveHybrid(threshold_gc_to_fo=0.2, threshold_fo_to_gc=0.05, dtmax=T, dtmin=1.0e-4 * T,
                            check_interval=50, save_adiabaticity=False)
    for kw in (dict(), dict(save_start=False), dict(save_everystep=False), dict(savestepinterval=7, save_end=False)):
        sols, r, a = _both(tp, orc, prob, alg, **kw)
        assert a is None and sols.adiabaticity is None
        _check(sols, r, None)


def test_hybrid_forced_fo_is_boris_on_gpu(tp, orc):
    B0 = 0.01
    q2m = tp.qi / tp.mi
    T = 2 * math.pi / (abs(q2m) * B0)
    rng = np.random.default_rng(2)
    u0 = np.zeros((6, 64))
    u0[3:] = rng.normal(0, 5.0e4, (3, 64))
    p = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, B0)), species=tp.Proton)
    alg = tp.AdaptiveHybrid(threshold=0.0, dtmax=10 * T, dtmin=1.0e-6 * T, check_interval=100)
    sols, r, a = _both(tp, orc, tp.TraceHybridProblem(u0, (0.0, 30 * T), p), alg)
    _check(sols, r, a, tol=1e-13)
    dt_fo = 2 * math.pi * alg.safety_fo / (abs(q2m) * B0)
    sb = tp.solve(tp.TraceProblem(u0, (0.0, 30 * T), p), tp.Boris(), dt=dt_fo)
    assert np.array_equal(sb.nsaved, sols.nsaved)
    for i in range(64):
        h, b = sols[i], sb[i]
        for k in range(len(b.t)):
            uu = h(b.t[k])
            assert np.linalg.norm(uu[:3] - b.u[k, :3]) <= 1.0e-8
            assert np.linalg.norm(uu[3:] - b.u[k, 3:]) <= 1.0e-5


def test_hybrid_dipole_and_grid_fields(tp, orc):
    # 1 keV - 10 MeV protons at 3 - 7 R_E in the Earth dipole: GC for the cold
    # ones, full orbit for the hot ones; then the same on a cubic grid of the field
    rng = np.random.default_rng(7)
    n = 128
    r = rng.uniform(3.0, 7.0, n) * tp.Re
    th = rng.uniform(0.4 * math.pi, 0.6 * math.pi, n)
    ph = rng.uniform(0, 2 * math.pi, n)
    x = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)])
    Ek = np.exp(rng.uniform(math.log(1.0e3), math.log(1.0e7), n))
    vmag = np.array([tp.energy2velocity(e) for e in Ek])
    d = rng.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    u0 = np.concatenate([x, vmag * d])
    B = tp.DipoleField(tp.BMoment_Earth)
    alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=1.0, dtmin=1.0e-4, check_interval=20, maxiters=4000)
    prob = tp.TraceHybridProblem(u0, (0.0, 60.0), tp.prepare(tp.ZeroField(), B, species=tp.Proton))
    sols, rr, a = _both(tp, orc, prob, alg, savestepinterval=50,
                        isoutside=tp.TerminateShell(1.5 * tp.Re, 12 * tp.Re))
    _check(sols, rr, a)
    assert set(sols.adiabaticity[2][:, 1]) == {0.0, 1.0}
    # a cubic grid of a quadratic field (the general-grid path)
    qf = tp.QuadraticField.bottle(1.0e-4, 1.0e-2)
    g = np.linspace(-40.0, 40.0, 33)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    A = np.stack([qf(np.array([xx, yy, zz])) for xx, yy, zz in zip(X.ravel(), Y.ravel(), Z.ravel())], axis=1)
    A = A.reshape(3, 33, 33, 33)
    Bg = tp.build_interpolator(A, g, g, g, 3)
    prob, T = _bottle(tp, n=64, seed=9)
    u0 = np.array(prob.u0)
    u0[5] *= 0.2   # mirror inside the grid
    prob = tp.TraceHybridProblem(u0, (0.0, 10 * T), tp.prepare(tp.ZeroField(), Bg, species=tp.Proton))
    alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=T, dtmin=1.0e-4 * T, check_interval=100)
    sols, rr, a = _both(tp, orc, prob, alg, savestepinterval=10)
    _check(sols, rr, a)
