"""Pin the CPU oracle to the reference's own known-answer tests.

Every expected number below is quoted from the reference test suite
(TestParticle.jl v0.23.2, test/...); the oracle restates the reference
solver, so these checks are what makes it a trustworthy checker for the
CUDA library.  Julia closures of those tests become Python callables passed
to the oracle as C callbacks.  No GPU needed.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import julia_isapprox


def _solve(tp, orc, u0, tspan, param, alg, E=None, B=None, isoutside=None, trajectories=1,
           prob_func=None, **kw):
    """Oracle solve of a TraceProblem; E/B override the param fields with callables."""
    q2m, m, Ep, Bp, F = param
    place = (q2m, m, tp.ZeroField(), tp.ZeroField(), F)
    prob = tp.TraceProblem(u0, tspan, place, prob_func=prob_func)
    plan = tp.plan_boris(prob, alg, tp.EnsembleB200(), trajectories=trajectories, **kw)
    return orc.boris_run(plan.desc, E if E is not None else Ep, B if B is not None else Bp, plan.u0,
                         plan.dt_i, plan.tend_i, isoutside=isoutside)


# ------------------------------------------------------------------ test/test_boris.jl
def test_basic_boris_final_state_and_interpolation(tp, orc):
    # test_boris.jl:40-61
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param, tp.Boris(),
               dt=3.0e-11, savestepinterval=10)
    t, u = r.traj(0)
    assert julia_isapprox(u[-1], [-0.00010199137926394769, 3.46340469171306e-5, 0.0,
                                  -60893.043824907196, -79322.36263335795, 0.0])
    assert t.size == u.shape[0]
    sol = tp.TraceSolution(t, u, "Success", "boris")
    assert julia_isapprox(sol(3.0e-8 / 2), [-3.8587882024745045e-5, 5.3855907133664956e-5, 0.0,
                                            -94689.58829601014, 32154.033469101283, 0.0])


def test_basic_boris_ensembles(tp, orc):
    # test_boris.jl:63-78 (prob_func sets vy = sim_id * 1e5)
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)

    def pf(prob, ctx):
        u = list(prob.u0)
        u[4] = ctx.sim_id * 1.0e5
        return tp.remake(prob, u0=u)

    r = _solve(tp, orc, [0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param, tp.Boris(),
               dt=3.0e-11, savestepinterval=1000, trajectories=4, prob_func=pf)
    assert julia_isapprox(r.final_states()[:, 3].sum(), -608930.4382490724)
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param, tp.Boris(),
               dt=3.0e-11, savestepinterval=1000, trajectories=2, prob_func=pf)
    assert julia_isapprox(r.final_states().sum(), -420646.2195768674)


def test_time_varying_field_accumulated_time(tp, orc):
    # test_boris.jl:80-88: the field depends on t, which pins the accumulated-time rule
    def B(x, t):
        if x[0] > 100 * t:
            bz = 1.0e-8
        elif x[0] < -10.0:
            bz = 1.0e-8
        else:
            bz = 0.0
        return (0.0, 0.0, bz)

    param = tp.prepare(tp.ZeroField(), tp.ZeroField(), species=tp.Electron)
    r = _solve(tp, orc, [-1.0, 0.0, 0.0, 1.0e6, 0.0, 0.0], (0.0, 0.01), param, tp.Boris(), B=B,
               dt=1.0e-4, savestepinterval=100)
    assert julia_isapprox(r.final_states()[0, 0], -512.8807214528281)


@pytest.mark.parametrize("alg", ["boris", "ms2n2", "h4n2", "h6n2", "h4n1"])
def test_multistep_exb_drift(tp, orc, alg):
    # test_boris.jl:95-125,162-188: E x B drift reaches x = 10 at t = 10
    algs = {"boris": tp.Boris(), "ms2n2": tp.MultistepBoris(2, 2), "h4n2": tp.MultistepBoris(4, 2),
            "h6n2": tp.MultistepBoris(6, 2), "h4n1": tp.MultistepBoris(4, 1)}
    param = (1.0, 1.0, tp.UniformField((0.0, 1.0, 0.0)), tp.UniformField((0.0, 0.0, 1.0)), tp.ZeroField())
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0.0, 10.0), param, algs[alg], dt=0.1)
    end = r.final_states()[0]
    assert abs(end[0] - 10.0) <= 1e-6
    assert abs(end[3] - 1.0) <= 1e-6


@pytest.mark.parametrize("alg", ["boris", "ms2n2", "ms2n4", "h4n4", "h6n4"])
def test_multistep_gyration_closes(tp, orc, alg):
    # test_boris.jl:127-159,190-209
    algs = {"boris": tp.Boris(), "ms2n2": tp.MultistepBoris(2, 2), "ms2n4": tp.MultistepBoris(2, 4),
            "h4n4": tp.MultistepBoris(4, 4), "h6n4": tp.MultistepBoris(6, 4)}
    param = (1.0, 1.0, tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0)), tp.ZeroField())
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0.0, 2 * math.pi), param, algs[alg], dt=0.1)
    end = r.final_states()[0]
    assert math.hypot(*end[:3]) < 0.02
    assert abs(math.hypot(*end[3:6]) - 1.0) <= 2.0e-3


def test_adaptive_boris_shrinks_dt_and_conserves_energy(tp, orc):
    # test_boris.jl:212-248: B = (0, 0, 0.01 (1 + x)), E = (0, 1e5, 0), electron
    tperiod = abs(tp.get_gyroperiod(0.01, q=tp.qe, m=tp.me))
    E = tp.UniformField((0.0, 1.0e5, 0.0))
    B = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    param = tp.prepare(E, B, species=tp.Electron)
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0e7, 0.0, 0.0], (0.0, 200 * tperiod), param,
               tp.AdaptiveBoris(0.1))
    t, u = r.traj(0)
    dt_end = t[-2] - t[-3]
    dt_start = t[10] - t[9]
    assert dt_end < 0.8 * dt_start

    def energy(s):
        return 0.5 * tp.me * np.dot(s[3:6], s[3:6]) + tp.qe * (-1.0e5 * s[1])

    assert abs(energy(u[-1]) - energy(u[0])) <= 1.0e-3 * max(abs(energy(u[0])), abs(energy(u[-1])))


def test_nonzero_tspan_start(tp, orc):
    # test_boris.jl:250-272: B exists only for t > 5; tspan starts at 10
    def B(x, t):
        return (0.0, 0.0, 0.01) if t > 5 else (0.0, 0.0, 0.0)

    param = tp.prepare(tp.ZeroField(), tp.ZeroField())
    u0 = [0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0]
    r = _solve(tp, orc, u0, (10.0, 10.1), param, tp.Boris(), B=B, dt=0.001)
    assert abs(r.final_states()[0, 3]) < 1.0e5 - 100
    r = _solve(tp, orc, u0, (10.0, 10.1), param, tp.AdaptiveBoris(0.1), B=B)
    assert abs(r.final_states()[0, 3]) < 1.0e5 - 100


@pytest.mark.parametrize("flags,n_expected", [
    (dict(savestepinterval=10), 101),
    (dict(savestepinterval=10, save_everystep=False, save_start=False, save_end=True), 1),
    (dict(savestepinterval=10, save_everystep=False, save_start=True, save_end=True), 2),
    (dict(savestepinterval=10, save_everystep=False, save_start=True, save_end=False), 1),
    (dict(savestepinterval=10, save_everystep=True, save_start=False, save_end=False), 99),
    (dict(savestepinterval=3, save_everystep=True, save_start=True, save_end=True), 335),
])
def test_saving_flags(tp, orc, flags, n_expected):
    # test_boris.jl:274-346
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)
    dt = 3.0e-11
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param, tp.Boris(), dt=dt, **flags)
    t, u = r.traj(0)
    assert t.size == n_expected
    if flags.get("save_start", True):
        assert t[0] == 0.0
    if n_expected == 1 and not flags.get("save_start", True):
        assert t[0] == 3.0e-8
    if n_expected == 99:
        assert math.isclose(t[0], 10 * dt) and math.isclose(t[-1], 990 * dt)
    if n_expected == 335:
        assert math.isclose(t[1], 3 * dt) and math.isclose(t[-2], 999 * dt) and t[-1] == 3.0e-8
    if n_expected == 101:
        assert t[-1] == 3.0e-8


def test_saving_flags_multistep_and_fields(tp, orc):
    # test_boris.jl:348-371
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)
    u0 = [0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0]
    r = _solve(tp, orc, u0, (0.0, 3.0e-8), param, tp.MultistepBoris(2, 2), dt=3.0e-11, savestepinterval=10,
               save_everystep=False, save_start=True, save_end=True)
    t, _ = r.traj(0)
    assert t.size == 2 and t[0] == 0.0 and t[-1] == 3.0e-8
    r = _solve(tp, orc, u0, (0.0, 3.0e-8), param, tp.Boris(), dt=3.0e-11, savestepinterval=10, save_fields=True)
    _, u = r.traj(0)
    assert u.shape[1] == 12
    assert list(u[0, 6:9]) == [0.0, 0.0, 0.0] and list(u[0, 9:12]) == [0.0, 0.0, 0.01]
    assert list(u[-1, 6:9]) == [0.0, 0.0, 0.0] and list(u[-1, 9:12]) == [0.0, 0.0, 0.01]


def _work_fields(tp, rate=0.0):
    """constant_E / gradient_B / time_varying_B_linear of test_boris.jl:24-28,419-421."""
    E = tp.UniformField((0.0, 1.0e5, 0.0))
    Bgrad = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    Bbeta = tp.AffineField((0.0, 0.0, 0.01), rate=(0.0, 0.0, 0.01 * 1.0e7))
    return E, Bgrad, Bbeta


def test_save_work_kats(tp, orc):
    # test_boris.jl:374-466
    E, Bgrad, Bbeta = _work_fields(tp)
    u0 = [0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0]
    tspan, dt = (0.0, 1.0e-9), 1.0e-11
    param = tp.prepare(E, Bgrad, species=tp.Electron)
    r = _solve(tp, orc, u0, tspan, param, tp.Boris(), dt=dt, savestepinterval=1, save_work=True,
               save_everystep=True)
    _, u = r.traj(0)
    assert u.shape[1] == 10
    work = u[0, 6:10]
    assert abs(work[0]) <= 1e-10 and abs(work[1]) <= 1e-10 and abs(work[3]) <= 1e-10
    assert abs(work[2]) > 0.0
    # P_grad = mu/|B| (b x grad|B|) . E with mu = m vperp^2 / 2|B| at the start
    mu = tp.Electron.m * 1.0e10 / (2 * 0.01)
    assert math.isclose(work[2], mu / 0.01 * 0.01 * 1.0e5, rel_tol=1e-12)

    # betatron: B_z = 0.01 (1 + 1e7 t), E = 0
    rb = _solve(tp, orc, u0, tspan, tp.prepare(tp.ZeroField(), Bbeta, species=tp.Electron), tp.Boris(), dt=dt,
                savestepinterval=1, save_work=True)
    assert rb.traj(0)[1][0, 9] > 0.0
    # the same field as a Julia-style closure: dB/dt by the oracle's central difference
    rc = _solve(tp, orc, u0, tspan, tp.prepare(tp.ZeroField(), Bbeta, species=tp.Electron), tp.Boris(),
                B=lambda x, t: np.array([0.0, 0.0, 0.01 * (1.0 + 1.0e7 * t)]), dt=dt, savestepinterval=1,
                save_work=True)
    assert np.allclose(rc.traj(0)[1][:, 9], rb.traj(0)[1][:, 9], rtol=1e-6)

    # both flags: width 16, work after the fields and identical to the work-only run
    r2 = _solve(tp, orc, u0, tspan, param, tp.Boris(), dt=dt, savestepinterval=1, save_fields=True,
                save_work=True)
    _, u2 = r2.traj(0)
    assert u2.shape[1] == 16
    assert np.array_equal(u2[0, 12:16], u[0, 6:10])
    assert np.array_equal(u2[:, 12:16], u[:, 6:10])
    assert np.array_equal(u2[:, 6:9], np.tile([0.0, 1.0e5, 0.0], (u2.shape[0], 1)))

    # MultistepBoris{2}(n = 2)
    rm = _solve(tp, orc, u0, tspan, param, tp.MultistepBoris(2, 2), dt=dt, savestepinterval=1, save_work=True)
    _, um = rm.traj(0)
    assert um.shape[1] == 10 and abs(um[0, 6]) <= 1e-10 and abs(um[0, 8]) > 0.0

    # AdaptiveBoris(safety = 0.1)
    ra = _solve(tp, orc, u0, tspan, param, tp.AdaptiveBoris(0.1), save_work=True, save_everystep=True)
    _, ua = ra.traj(0)
    assert ua.shape[1] == 10 and abs(ua[0, 6]) <= 1e-10 and abs(ua[0, 8]) > 0.0


def test_gc_save_fields_and_work_kat(tp, orc):
    # test_gc.jl:268-304: fields and work saved by the guiding-centre solver
    B = tp.DipoleField(tp.BMoment_Earth)
    r0 = [1.5 * tp.Re, 0.0, 0.0]
    v0 = [0.0, 1.0e5, 1.0e5]
    q, m = tp.Proton.q, tp.Proton.m
    y, mu = orc.gc_prepare(tp.ZeroField(), B, np.array([r0 + v0]), q, m)
    y0, param = y[0], (q, q / m, float(mu[0]), tp.ZeroField(), B)
    prob = tp.TraceGCProblem(y0, (0.0, 1.0e-4), param)
    plan = tp.plan_gc(prob, tp.EnsembleB200(), trajectories=2, dt=1.0e-5, save_fields=True, save_work=True)
    r = orc.gc_run(plan.desc, plan.E, plan.B, plan.y0)
    for i in range(2):
        t, u = r.traj(i)
        assert u.shape == (t.size, 14)
        assert np.linalg.norm(u[0, 7:10]) > 0.0
        assert np.linalg.norm(u[0, 4:7]) == 0.0
        # E = 0: every electric work term vanishes; static B: no betatron term
        assert np.all(u[:, 10:14] == 0.0)


def test_solver_limits(tp, orc):
    # test_boris.jl:509-532
    E = tp.UniformField((0.0, 1.0e5, 0.0))
    B = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    param = tp.prepare(E, B, species=tp.Electron)
    u0 = [0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0]
    with pytest.raises(ValueError):
        _solve(tp, orc, u0, (0.0, 1.0e-9), param, tp.Boris(), dt=1.0e-11, maxiters=50)
    with pytest.raises(ValueError):
        _solve(tp, orc, u0, (0.0, 1.0e-9), param, tp.Boris(), dt=np.finfo(float).eps)
    with pytest.raises(ValueError):
        tp.MultistepBoris(1)
    with pytest.raises(ValueError):
        tp.MultistepBoris(3, 2)


# ------------------------------------------------------------------ test/test_boris_kernel.jl
def test_energy_conservation_two_periods(tp, orc):
    # test_boris_kernel.jl:95-116
    B0 = 1.0e-8
    T = 2 * math.pi / (tp.qi * B0 / tp.mi)
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, B0)), species=tp.Proton)
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0], (0.0, 2 * T), param, tp.Boris(), dt=T / 100,
               savestepinterval=10)
    v = r.final_states()[0, 3:6]
    assert abs(np.linalg.norm(v) - 1.0e5) <= 1.0e-3 * 1.0e5


# ------------------------------------------------------------------ test/test_adaptive_multistep_boris.jl
def test_adaptive_multistep_n1_matches_adaptive_boris(tp, orc):
    # test_adaptive_multistep_boris.jl:41-48
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0e-8)))
    u0 = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0]
    a = _solve(tp, orc, u0, (0.0, 1.0), param, tp.AdaptiveBoris(0.1))
    b = _solve(tp, orc, u0, (0.0, 1.0), param, tp.AdaptiveMultistepBoris(2, 1, 0.1))
    assert julia_isapprox(a.t, b.t)
    assert julia_isapprox(a.u, b.u)
    assert a.retcode[0] == 1 and b.retcode[0] == 1


# ------------------------------------------------------------------ test/test_boundary.jl
def _nan_fields():
    def E(r, t):
        return (math.nan,) * 3 if np.linalg.norm(r) > 1.0 else (0.0, 0.0, 0.0)

    def B(r, t):
        return (math.nan,) * 3 if np.linalg.norm(r) > 1.0 else (0.0, 0.0, 1.0)

    def isoutside(u, t):
        return bool(np.any(np.isnan(u))) or np.linalg.norm(u[:3]) > 1.0

    return E, B, isoutside


def test_boundary_nan_boris_and_adaptive(tp, orc):
    # test_boundary.jl:10-58
    E, B, out = _nan_fields()
    p = (1.0, 1.0, tp.ZeroField(), tp.ZeroField(), tp.ZeroField())
    u0 = [0.9, 0.0, 0.0, 0.0, 1.0, 0.0]
    for alg, kw in ((tp.Boris(), dict(dt=0.2)), (tp.AdaptiveBoris(0.05), {})):
        r = _solve(tp, orc, u0, (0.0, 1.0), p, alg, E=E, B=B, isoutside=out, **kw)
        end = r.final_states()[0]
        assert not np.any(np.isnan(end))
        assert np.linalg.norm(end[:3]) <= 1.0
        assert r.retcode[0] == 2  # Terminated


def _gc_solve(tp, orc, y0, tspan, p, E=None, B=None, isoutside=None, **kw):
    q, q2m, mu, Ep, Bp = p
    prob = tp.TraceGCProblem(y0, tspan, (q, q2m, mu, tp.ZeroField(), tp.ZeroField()))
    plan = tp.plan_gc(prob, tp.EnsembleB200(), **kw)
    return orc.gc_run(plan.desc, E if E is not None else Ep, B if B is not None else Bp, plan.y0,
                      isoutside=isoutside)


def test_boundary_nan_gc(tp, orc):
    # test_boundary.jl:60-81
    E, B, out = _nan_fields()
    p = (1.0, 1.0, 0.0, None, None)
    for kw in (dict(dt=0.2, alg="rk4"), dict(dt=0.01, alg="rk45")):
        r = _gc_solve(tp, orc, [0.9, 0.0, 0.0, 1.0], (0.0, 1.0), p, E=E, B=B, isoutside=out, **kw)
        end = r.final_states()[0]
        assert not np.any(np.isnan(end))
        assert np.linalg.norm(end[:3]) <= 1.0
        assert r.retcode[0] == 2


def test_boundary_spatial_and_time_rejection(tp, orc):
    # test_boundary.jl:84-128
    param = tp.prepare(tp.ZeroField(), tp.UniformField((1.0, 0.0, 0.0)), species=tp.Proton)
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0], (0.0, 1.0e-5), param, tp.AdaptiveBoris(0.1),
               isoutside=lambda u, t: u[0] > 0.5)
    t, u = r.traj(0)
    assert u[-1, 0] <= 0.5 and t[-1] < 1.0e-5 and r.retcode[0] == 2
    # integer tspan
    r = _solve(tp, orc, [0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0, 10), param, tp.Boris(), dt=1.0)
    t, _ = r.traj(0)
    assert t[-1] == 10 and r.retcode[0] == 1
    # GC time rejection
    Eg, Bg = tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0))
    y0, mu = orc.gc_prepare(Eg, Bg, np.array([0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0]), tp.qi, tp.mi)
    p = (tp.qi, tp.qi / tp.mi, mu[0], Eg, Bg)
    r = _gc_solve(tp, orc, y0[0], (0.0, 1.0), p, dt=1.0e-4, alg="rk4", isoutside=lambda u, t: t > 0.5)
    t, _ = r.traj(0)
    assert math.isclose(t[-1], 0.5, rel_tol=1e-8) and r.retcode[0] == 2


# ------------------------------------------------------------------ test/test_gc.jl
def _gc_dipole_problem(tp, orc):
    # test_gc.jl:166-186: 50 MeV proton at 2.5 R_E in the Earth dipole
    Ek = 5.0e7
    v0 = tp.sph2cart(tp.energy2velocity(Ek, m=tp.mi, q=tp.qi), math.pi / 4, 0.0)
    r0 = tp.sph2cart(2.5 * tp.Re, math.pi / 2, 0.0)
    E = tp.ZeroField()
    B = tp.DipoleField(tp.BMoment_Earth)
    y0, mu = orc.gc_prepare(E, B, np.concatenate([r0, v0]), tp.qi, tp.mi)
    return y0[0], (tp.qi, tp.qi / tp.mi, mu[0], E, B)


def test_gc_rk4_dipole_counts(tp, orc):
    y0, p = _gc_dipole_problem(tp, orc)
    r = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk4")
    assert r.nsaved[0] == 10001 and r.retcode[0] == 3  # MaxIters
    r = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk4", save_everystep=False)
    assert r.nsaved[0] == 2
    r = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk4", isoutside=lambda u, t: t > 0.5)
    assert r.nsaved[0] == 5001


def test_gc_rk45_dipole_counts(tp, orc):
    y0, p = _gc_dipole_problem(tp, orc)
    r = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk45")
    assert r.nsaved[0] == 61 and r.retcode[0] == 1
    tight = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk45", abstol=1e-8, reltol=1e-8)
    assert tight.nsaved[0] > 61
    rk4 = _gc_solve(tp, orc, y0, (0.0, 1.0), p, dt=1.0e-4, alg="rk4")
    assert np.linalg.norm(tight.final_states()[0] - rk4.final_states()[0]) < 10.0
    auto = _gc_solve(tp, orc, y0, (0.0, 1.0), p, alg="rk45")
    assert auto.nsaved[0] == 58 and auto.retcode[0] == 1


def test_gc_full_conversion_kats(tp, orc):
    """test_gc.jl:62-160: GC -> full -> GC reversibility, the E x B drift and the gyrophase."""
    q, m = tp.Proton.q, tp.Proton.m
    Z, B1 = tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0))
    R, vpar, mu = np.array([1.0, 0.0, 0.0]), 1.0e5, 1.0e-15
    xu = orc.gc_to_full(Z, B1, np.r_[R, vpar], mu, q, m, np.pi / 3)[0]
    assert xu.shape == (6,)
    y, mu_new = orc.gc_prepare(Z, B1, xu, q, m)
    assert np.allclose(y[0, :3], R, rtol=1e-5) and np.isclose(y[0, 3], vpar, rtol=1e-5)
    assert np.isclose(mu_new[0], mu, rtol=1e-5)
    # E in y, B in z: the drift (E x B) / B^2 = (1000, 0, 0)
    E2 = tp.UniformField((0.0, 1.0e3, 0.0))
    xu = orc.gc_to_full(E2, B1, np.zeros(4), 0.0, q, m)[0]
    assert np.allclose(xu[3:], [1000.0, 0.0, 0.0], atol=1e-5)
    y, mu_new = orc.gc_prepare(E2, B1, xu, q, m)
    assert np.allclose(y[0], 0.0, atol=1e-5) and abs(mu_new[0]) <= 1e-10
    # phase 0 along e1 = x, phase pi/2 along e2 = y (get_perp_vector of z)
    v0 = orc.gc_to_full(Z, B1, np.zeros(4), 1.0e-15, q, m, 0.0)[0, 3:]
    v90 = orc.gc_to_full(Z, B1, np.zeros(4), 1.0e-15, q, m, np.pi / 2)[0, 3:]
    n0, n90 = v0 / np.linalg.norm(v0), v90 / np.linalg.norm(v90)
    assert abs(n0 @ n90) <= 1e-5
    assert np.allclose(n0, [1.0, 0.0, 0.0], atol=1e-5) and np.allclose(n90, [0.0, 1.0, 0.0], atol=1e-5)


# ------------------------------------------------------------------ test/test_utility.jl
def test_gyro_constants(tp):
    # test_utility.jl:28-33
    assert math.isclose(tp.get_gyroradius(440.0e3, 5.0e-9), 918692.2725070775, rel_tol=1.5e-8)
    assert math.isclose(tp.get_gyroperiod(5.0e-9), 13.118894973717941, rel_tol=1.5e-8)


def _scalar_grid(tp, bc, order=1):
    # test_utility.jl:93-110: n[i,j,k] = i + j + k (1-based) on x(4), y(6), z(8) in [-10, 10]
    x = np.linspace(-10, 10, 4)
    y = np.linspace(-10, 10, 6)
    z = np.linspace(-10, 10, 8)
    i, j, k = np.meshgrid(np.arange(1, 5), np.arange(1, 7), np.arange(1, 9), indexing="ij")
    A = (i + j + k).astype(np.float32)   # a scalar grid: carried as component 0
    return tp.build_interpolator(A, x, y, z, order, bc)


def test_interpolation_kats(tp, orc):
    f = _scalar_grid(tp, tp.FillExtrap())
    assert math.isclose(orc.field_eval(f, [9.0, 0.0, 0.0])[0, 0], 11.85, rel_tol=1e-12)
    assert np.all(np.isnan(orc.field_eval(f, [20.0, 0.0, 0.0])))
    f = _scalar_grid(tp, tp.PeriodicBC("exclusive"))
    assert math.isclose(orc.field_eval(f, [20.0, 0.0, 0.0])[0, 0], 9.5, rel_tol=1e-12)
    f = _scalar_grid(tp, tp.ClampExtrap())
    assert math.isclose(orc.field_eval(f, [20.0, 0.0, 0.0])[0, 0], 12.0, rel_tol=1e-12)


def test_interpolation_order0_and_cubic_kats(tp, orc):
    # test_utility.jl:103-120: constant (order 0) and cardinal cubic (order 3)
    f = _scalar_grid(tp, tp.FillExtrap(), order=0)
    assert math.isclose(orc.field_eval(f, [-10.0, -10.0, -10.0])[0, 0], 3.0, rel_tol=1e-12)
    f = _scalar_grid(tp, tp.FillExtrap(), order=3)
    assert math.isclose(orc.field_eval(f, [9.0, 0.0, 0.0])[0, 0], 11.85, rel_tol=1e-12)
    f = _scalar_grid(tp, tp.PeriodicBC("exclusive"), order=3)
    assert math.isclose(orc.field_eval(f, [20.0, 0.0, 0.0])[0, 0], 9.25, rel_tol=1e-12)
    f = _scalar_grid(tp, tp.ClampExtrap(), order=3)
    assert math.isclose(orc.field_eval(f, [20.0, 0.0, 0.0])[0, 0], 12.0, rel_tol=1e-12)
    # the cubic passes through the nodes and reproduces quadratics inside
    x = np.linspace(0.0, 1.0, 9)
    A = np.zeros((3, 9, 9, 9))
    A[0] = (x ** 2)[:, None, None] + 0 * x[None, :, None] + 0 * x[None, None, :]
    g = tp.build_interpolator(A, x, x, x, 3)
    assert math.isclose(orc.field_eval(g, [0.375, 0.5, 0.5])[0, 0], 0.375 ** 2, rel_tol=1e-12)
    assert math.isclose(orc.field_eval(g, [0.4, 0.5, 0.5])[0, 0], 0.16, rel_tol=1e-12)
    assert math.isclose(orc.field_eval(g, [0.05, 0.5, 0.5])[0, 0], 0.0025, rel_tol=1e-12)


def _spherical_br(tp, r, order):
    th = np.linspace(0, math.pi, 11)
    ph = np.linspace(0, 2 * math.pi, 11)
    B = np.zeros((3, len(r), 11, 11))
    B[0] = 1.0
    return tp.build_interpolator(tp.StructuredGrid, B, r, th, ph, order)


def test_spherical_interpolation_kats(tp, orc):
    # test_utility.jl:123-166: B_r = 1 gives the unit radial vector
    for r in (np.linspace(0.1, 10, 11), np.geomspace(1.0, 10.0, 11)):
        for order in (0, 1, 3) if r[0] == 0.1 else (1,):
            B = _spherical_br(tp, r, order)
            v = orc.field_eval(B, [1.0, 1.0, 1.0])[0]
            assert np.allclose(v, [0.57735] * 3, atol=1e-5)
        A = np.ones((len(r), 11, 11))
        f = tp.build_interpolator(tp.StructuredGrid, A, r, np.linspace(0, math.pi, 11),
                                  np.linspace(0, 2 * math.pi, 11))
        assert orc.field_eval(f, [1.0, 1.0, 1.0])[0, 0] == 1.0
        assert np.isnan(orc.field_eval(f, [0.0, 0.0, 0.0])[0, 0])


def test_rectilinear_interpolation_kats(tp, orc):
    # test_utility.jl:259-314 (CartesianNonUniform)
    x = np.linspace(0.0, 10.0, 11)
    B = np.zeros((3, 11, 11, 11))
    B[0] = 1.0
    f = tp.build_interpolator(tp.RectilinearGrid, B, x, x, x)
    assert np.allclose(orc.field_eval(f, [5.0, 5.0, 5.0])[0], [1.0, 0.0, 0.0])
    i, j, k = np.meshgrid(x, x, x, indexing="ij")
    f = tp.build_interpolator(tp.RectilinearGrid, i + j + k, x, x, x)
    assert math.isclose(orc.field_eval(f, [5.0, 5.0, 5.0])[0, 0], 15.0, rel_tol=1e-12)
    assert math.isclose(orc.field_eval(f, [5.5, 5.5, 5.5])[0, 0], 16.5, rel_tol=1e-12)
    xn = np.array([0.0, 1.0, 4.0, 9.0])
    i, j, k = np.meshgrid(xn, xn, xn, indexing="ij")
    f = tp.build_interpolator(tp.RectilinearGrid, np.sqrt(i) + np.sqrt(j) + np.sqrt(k), xn, xn, xn)
    assert math.isclose(orc.field_eval(f, [4.0, 4.0, 4.0])[0, 0], 6.0, rel_tol=1e-12)
    assert math.isclose(orc.field_eval(f, [1.0, 4.0, 9.0])[0, 0], 6.0, rel_tol=1e-12)


@pytest.mark.parametrize("dims", [3, 2, 1])
def test_grid_jacobians_match_finite_differences(tp, orc, dims):
    # test_derivatives.jl:6-50 (1-D / 2-D / 3-D), plus the cubic and spherical grids
    rng = np.random.default_rng(3)
    x = np.linspace(0.0, 1.0, 5)
    shape = (3,) + (5,) * dims
    A = rng.normal(size=shape)
    fields = [tp.build_interpolator(tp.CartesianGrid, A, *([x] * dims), order) for order in (1, 3)]
    if dims == 3:
        r, th, ph = np.linspace(0.5, 2.0, 7), np.linspace(0, math.pi, 9), np.linspace(0, 2 * math.pi, 13)
        fields += [tp.build_interpolator(tp.StructuredGrid, rng.normal(size=(3, 7, 9, 13)), r, th, ph, o)
                   for o in (1, 3)]
    p = np.array([0.43, 0.61, 0.27])
    for f in fields:
        _, J = orc.field_eval(f, p, jacobian=True)
        h = 1e-6
        for c in range(3):
            e = np.zeros(3)
            e[c] = h
            fd = (orc.field_eval(f, p + e) - orc.field_eval(f, p - e))[0] / (2 * h)
            assert np.allclose(J[0][:, c], fd, rtol=1e-6, atol=1e-8)
        if dims < 3:   # unused coordinates have zero derivative
            assert np.all(J[0][:, dims:] == 0.0)


def test_dipole_jacobian_matches_finite_differences(tp, orc):
    B = tp.DipoleField(tp.BMoment_Earth)
    x = np.array([2.1 * tp.Re, 0.7 * tp.Re, 0.4 * tp.Re])
    _, J = orc.field_eval(B, x, jacobian=True)
    h = 1.0
    for jdx in range(3):
        e = np.zeros(3)
        e[jdx] = h
        fd = (orc.field_eval(B, x + e) - orc.field_eval(B, x - e))[0] / (2 * h)
        assert np.allclose(J[0][:, jdx], fd, rtol=1e-6, atol=1e-20)


# ------------------------------------------------------------------ test/test_hybrid.jl
def _hybrid(tp, orc, u0, tspan, E, B, alg, species=None, **kw):
    q2m, m = tp.qi / tp.mi, tp.mi
    prob = tp.TraceHybridProblem(u0, tspan, (q2m, m, tp.ZeroField(), tp.ZeroField(), tp.ZeroField()))
    plan = tp.plan_hybrid(prob, alg, **kw)
    return orc.hybrid_run(plan.desc, E, B, plan.u0)


def test_hybrid_uniform_and_sheared_kats(tp, orc):
    # test_hybrid.jl:14-53
    u0 = [0.0, 0.0, 0.0, 1.0e4, 0.0, 1.0e3]
    alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=1.0e-6)
    r, a = _hybrid(tp, orc, u0, (0.0, 1.0e-4), tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), alg)
    assert r.retcode[0] == 1
    assert set(np.asarray(a.u)[:, 1]) == {0.0}   # uniform field: GC throughout
    B0, k = 0.01, 100.0

    def sheared(x, t):
        return (B0 * math.cos(k * x[0]), B0 * math.sin(k * x[0]), 0.0)

    def sheared_jac(x, t):
        return [[-B0 * k * math.sin(k * x[0]), 0, 0], [B0 * k * math.cos(k * x[0]), 0, 0], [0, 0, 0]]

    r, a = _hybrid(tp, orc, u0, (0.0, 1.0e-5), tp.ZeroField(), (sheared, sheared_jac), alg)
    assert r.retcode[0] == 1


def _bottle_case(tp):
    B0, alpha = 1.0e-4, 1.0e-2
    q2m = tp.qi / tp.mi
    T = 2 * math.pi / (abs(q2m) * B0)
    return tp.QuadraticField.bottle(B0, alpha), T


@pytest.mark.parametrize("buffer", [False, True])
def test_hybrid_bottle_switching_kat(tp, orc, buffer):
    # test_hybrid.jl:55-100,177-206
    B, T = _bottle_case(tp)
    u0 = [0.0, 0.0, 0.0, 5.0e4, 0.0, 1.0e5]
    if buffer:
        alg = tp.AdaptiveHybrid(threshold_gc_to_fo=0.2, threshold_fo_to_gc=0.05, dtmax=T, dtmin=1.0e-4 * T,
                                check_interval=100)
    else:
        alg = tp.AdaptiveHybrid(threshold=0.1, dtmax=T, dtmin=1.0e-4 * T, check_interval=100)
    r, a = _hybrid(tp, orc, u0, (0.0, 30 * T), tp.ZeroField(), B, alg)
    t, u = r.traj(0)
    assert r.retcode[0] == 1 and t.size > 100
    ke0 = 0.5 * tp.mi * (5.0e4 ** 2 + 1.0e5 ** 2)
    ke1 = 0.5 * tp.mi * np.sum(u[-1, 3:6] ** 2)
    assert abs(ke1 - ke0) <= 0.1 * ke0
    if not buffer:
        modes = set(np.asarray(a.u)[:, 1])
        assert modes == {0.0, 1.0}   # both modes visited


def test_hybrid_gc_roundtrip_exact_in_uniform_field(tp, orc):
    # test_hybrid.jl:102-121
    B = tp.UniformField((0.0, 0.0, 0.01))
    xv = np.array([[*x0, *v0] for x0 in ([0, 0, 0], [1.0, 0.5, 1.0], [3.0, 0, 2.0])
                   for v0 in ([5.0e4, 0, 1.0e5], [3.0e4, 4.0e4, 8.0e4])], dtype=float)
    rec = orc.gc_roundtrip(tp.ZeroField(), B, xv, tp.qi, tp.mi)
    assert np.all(np.linalg.norm(rec[:, :3] - xv[:, :3], axis=1) < 1.0e-10)
    assert np.all(np.linalg.norm(rec[:, 3:] - xv[:, 3:], axis=1) < 1.0e-8)


def test_hybrid_forced_fo_is_boris(tp, orc):
    # test_hybrid.jl:123-152: threshold 0 keeps the full orbit; it is Boris with dt_fo
    B0 = 0.01
    q2m = tp.qi / tp.mi
    T = 2 * math.pi / (abs(q2m) * B0)
    u0 = [0.0, 0.0, 0.0, 5.0e4, 0.0, 1.0e5]
    alg = tp.AdaptiveHybrid(threshold=0.0, dtmax=10 * T, dtmin=1.0e-6 * T, check_interval=100)
    r, _ = _hybrid(tp, orc, u0, (0.0, 30 * T), tp.ZeroField(), tp.UniformField((0.0, 0.0, B0)), alg)
    th, uh = r.traj(0)
    dt_fo = 2 * math.pi * alg.safety_fo / (abs(q2m) * B0)
    prob = tp.TraceProblem(u0, (0.0, 30 * T), (q2m, tp.mi, tp.ZeroField(), tp.ZeroField(), tp.ZeroField()))
    plan = tp.plan_boris(prob, tp.Boris(), dt=dt_fo)
    rb = orc.boris_run(plan.desc, tp.ZeroField(), tp.UniformField((0.0, 0.0, B0)), plan.u0)
    tb, ub = rb.traj(0)
    assert th.size == tb.size
    sol = tp.TraceSolution(th, uh, "Success", "hybrid")
    for i in range(tb.size):
        uu = sol(tb[i])
        assert np.linalg.norm(uu[:3] - ub[i, :3]) <= 1.0e-8
        assert np.linalg.norm(uu[3:] - ub[i, 3:]) <= 1.0e-5


def test_hybrid_argument_errors(tp):
    # test_hybrid.jl:154-175
    assert tp.AdaptiveHybrid(threshold=0.1, dtmax=1.0).threshold_gc_to_fo == 0.1
    assert tp.AdaptiveHybrid(threshold=0.1, dtmax=1.0).threshold_fo_to_gc == 0.1
    with pytest.raises(ValueError):
        tp.AdaptiveHybrid(threshold_gc_to_fo=0.05, threshold_fo_to_gc=0.2, dtmax=1.0)
    a = tp.AdaptiveHybrid(threshold_gc_to_fo=0.2, threshold_fo_to_gc=0.05, dtmax=1.0)
    assert a.threshold_gc_to_fo == 0.2 and a.threshold_fo_to_gc == 0.05
    with pytest.raises(ValueError):
        tp.AdaptiveHybrid(dtmax=1.0, check_interval=0)
    with pytest.raises(ValueError):
        tp.AdaptiveHybrid(dtmax=1.0, adiabaticity="nope")


def test_quadratic_field_matches_numpy(tp, orc):
    B = tp.QuadraticField.bottle(1.0e-4, 1.0e-2)
    pts = np.random.default_rng(1).normal(size=(50, 3)) * 10
    v, J = orc.field_eval(B, pts, jacobian=True)
    for i, x in enumerate(pts):
        assert np.allclose(v[i], B(x), rtol=1e-14, atol=0)
        h = 1e-5
        fd = np.stack([(B(x + h * e) - B(x - h * e)) / (2 * h) for e in np.eye(3)], axis=1)
        assert np.allclose(J[i], fd, rtol=1e-7, atol=1e-12)


def test_portable_gyrophase_trig_accuracy(orc):
    # the hybrid's sin / cos / atan2 (+, -, *, /, sqrt only, shared by the
    # kernel and the oracle): within 1 ulp of 1 and 4 ulp of pi of libm
    rng = np.random.default_rng(0)
    x = np.concatenate([np.linspace(-8, 8, 100001), rng.uniform(-8, 8, 100000), rng.normal(size=50000)])
    y = rng.normal(size=x.size)
    s, c, a = orc.trig(x, y)
    assert np.max(np.abs(s - np.sin(x))) <= np.spacing(1.0)
    assert np.max(np.abs(c - np.cos(x))) <= np.spacing(1.0)
    assert np.max(np.abs(a - np.arctan2(y, x))) <= 4 * np.spacing(np.pi)


def test_portable_trig_relative_accuracy_on_the_multistep_range(orc):
    # The closed-form MultistepBoris rotation (multistep_boris.jl:110-119)
    # calls atan(|t_n|) for |t_n| >= 1e-4 and sincos(n * alpha); the float64
    # kernel and the oracle both use the portable routines there.  Relative
    # error against libm: atan within 2 ulp up to tan(pi/16) (no half-angle
    # reduction: the typical |t_n| of a step), 4 ulp above; sin and cos
    # within 2 ulp of the larger of the value and 1e-3 (n * alpha lies in
    # (0, n * pi / 2)).
    rng = np.random.default_rng(1)
    t = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), 200000))
    _, _, a = orc.trig(np.ones_like(t), t)  # atan2(t, 1)
    ulps = np.abs(a - np.arctan(t)) / np.spacing(np.arctan(t))
    assert np.max(ulps[t <= 0.1989]) <= 2
    assert np.max(ulps) <= 4
    for n in (1, 2, 4, 6):
        x = n * np.arctan(t)
        s, c, _ = orc.trig(x, np.ones_like(x))
        assert np.max(np.abs(s - np.sin(x)) / np.spacing(np.maximum(np.abs(np.sin(x)), 1e-3))) <= 2
        assert np.max(np.abs(c - np.cos(x)) / np.spacing(np.maximum(np.abs(np.cos(x)), 1e-3))) <= 2


# ------------------------------------------------------------------ virtual detectors (test_utility.jl:768-960)
def _line(x0, y0, vx, vy, z0=0.0, vz=0.0, n=21):
    t = np.arange(float(n))
    u = np.stack([x0 + vx * t, y0 + vy * t, z0 + vz * t, np.full(n, vx), np.full(n, vy), np.full(n, vz)], axis=1)
    return t, u


def _pack_lines(*lines):
    t = np.concatenate([a for a, _ in lines])
    u = np.concatenate([b for _, b in lines])
    return t, u, np.array([len(a) for a, _ in lines], dtype=np.int32)


def test_detector_kats(tp, orc):
    disk = tp.Disk(tp.Plane((0.0, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    area = math.pi * 25.0
    l1 = _line(-10.0, 0.0, 1.0, 0.0)
    l2 = _line(-10.0, 10.0, 1.0, 0.0)      # misses the disk
    l3 = _line(5.0, -10.0, 0.0, 1.0)       # parallel to the plane
    sums, counts, rows, _ = orc.detect(*_pack_lines(l1), [disk])
    assert counts[0] == 1 and np.allclose(rows[0], [1.0, 0.0, 0.0, 1.0])
    assert math.isclose(sums[0, 0] / area, 1.0 / area) and np.allclose(sums[0, 1:] / area, [1.0 / area, 0, 0])
    for l in (l2, l3):
        sums, counts, _, _ = orc.detect(*_pack_lines(l), [disk])
        assert counts[0] == 0 and np.all(sums == 0.0)
    sums, counts, _, _ = orc.detect(*_pack_lines(l1, l2, l3), [disk], weights=[1.0, 2.0, 3.0])
    assert sums[0, 0] == 1.0
    sums, _, _, _ = orc.detect(*_pack_lines(l1, l1, l2), [disk], weights=[1.0, 2.0, 3.0])
    assert sums[0, 0] == 3.0 and np.allclose(sums[0, 1:], [3.0, 0.0, 0.0])
    _, counts, rows, _ = orc.detect(*_pack_lines(l1), [tp.Plane((0.0, 0.0, 0.0), (1.0, 0.0, 0.0))], weight=3.0)
    assert counts[0] == 1 and rows[0, 3] == 3.0 and np.allclose(rows[0, :3], [1.0, 0.0, 0.0])
    sums, counts, _, _ = orc.detect(*_pack_lines(l1), [tp.Sphere((0.0, 0.0, 0.0), 5.0)])
    assert counts[0] == 2 and np.allclose(sums[0], [2.0, 2.0, 0.0, 0.0])
    # equivalence: weight 2 at v = 1 and weight 1 at v = 2 (exact values)
    la, lb = _line(-10.0, 0.0, 1.0, 0.0), _line(-10.0, 0.0, 2.0, 0.0)
    _, _, ra, _ = orc.detect(*_pack_lines(la), [disk], weight=2.0)
    _, _, rb, _ = orc.detect(*_pack_lines(lb), [disk], weight=1.0)
    assert ra[0, 0] == 1.0 and ra[0, 3] == 2.0 and rb[0, 0] == 2.0 and rb[0, 3] == 1.0
    # two detectors on one segment (test_utility.jl:853-868)
    t = np.array([0.0, 2.0])
    u = np.array([[0.0, 0, 0, 1, 0, 0], [2.0, 0, 0, 1, 0, 0]])
    d1 = tp.Disk(tp.Plane((0.5, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    d2 = tp.Disk(tp.Plane((1.5, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    sums, counts, _, _ = orc.detect(t, u, [2], [d1, d2])
    assert list(counts) == [1, 1] and np.allclose(sums[:, :2], [[1.0, 1.0], [1.0, 1.0]])
    # first crossing (test_utility.jl:900-918)
    lz = _line(0.0, 0.0, 0.0, 0.0, z0=-10.0, vz=1.0)
    plane = tp.Plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    _, _, _, first = orc.detect(*_pack_lines(lz), [plane])
    assert np.allclose(first[0], [0, 0, 0, 0, 0, 1.0])
    _, _, _, first = orc.detect(*_pack_lines(lz), [tp.Plane((0.0, 0.0, 20.0), (0.0, 0.0, 1.0))])
    assert np.all(np.isnan(first[0]))


# ------------------------------------------------------------------ LazyTimeInterpolator
def test_lazy_time_interpolator_kats(tp, orc):
    # test_utility.jl:316-405: E = t * x snapshots at t = 0, 1, 2
    times = [0.0, 1.0, 2.0]
    itp = tp.LazyTimeInterpolator(times, lambda i: tp.AffineField((0.0, 0.0, 0.0), np.eye(3) * times[i - 1]))
    x = [1.0, 2.0, 3.0]
    for t, ref in [(0.0, [0, 0, 0]), (1.0, [1, 2, 3]), (0.5, [0.5, 1.0, 1.5]), (1.5, [1.5, 3.0, 4.5])]:
        assert np.allclose(orc.field_eval(itp, x, t)[0], ref, rtol=1e-14, atol=0)
    assert np.array_equal(orc.field_eval(itp, x, 3.0), orc.field_eval(itp, x, 2.0))
    assert np.array_equal(orc.field_eval(itp, x, -1.0), orc.field_eval(itp, x, 0.0))
    # numerical snapshots: B = (1, 0, 0) at t = 0, (0, 2, 0) at t = 1
    g = np.linspace(0.0, 1.0, 4)
    B0 = np.zeros((3, 4, 4, 4))
    B0[0] = 1.0
    B1 = np.zeros((3, 4, 4, 4))
    B1[1] = 2.0
    itp = tp.LazyTimeInterpolator([0.0, 1.0], lambda i: tp.build_interpolator(B0 if i == 1 else B1, g, g, g))
    pt = [0.5, 0.5, 0.5]
    for t, ref in [(0.0, [1, 0, 0]), (1.0, [0, 2, 0]), (0.5, [0.5, 1.0, 0]), (0.25, [0.75, 0.5, 0])]:
        assert np.allclose(orc.field_eval(itp, pt, t)[0], ref, rtol=1e-14, atol=1e-15)


def test_lazy_time_interpolator_derivatives(tp, orc):
    # test_derivatives.jl:57-90: Jacobian and d/dt against finite differences,
    # clamped Jacobians and zero d/dt outside the times
    times = [0.0, 1.0, 2.0]
    itp = tp.LazyTimeInterpolator(times, lambda i: tp.AffineField((0.0, 0.0, 0.0), np.eye(3) * times[i - 1]))
    pos = np.array([1.0, 2.0, 3.0])
    _, J = orc.field_eval(itp, pos, 0.5, jacobian=True)
    assert np.allclose(J[0], 0.5 * np.eye(3))
    _, Jm = orc.field_eval(itp, pos, -1.0, jacobian=True)
    _, J0 = orc.field_eval(itp, pos, 0.0, jacobian=True)
    _, J3 = orc.field_eval(itp, pos, 3.0, jacobian=True)
    _, J2 = orc.field_eval(itp, pos, 2.0, jacobian=True)
    assert np.array_equal(Jm, J0) and np.array_equal(J3, J2)
    # betatron work uses d|B|/dt: B(t) = t x along a unit x -> dB/dt = x inside, 0 outside
    B = tp.LazyTimeInterpolator(times, lambda i: tp.UniformField((0.0, 0.0, 1.0 + times[i - 1])))
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0.0, 0.5),
                           (1.0, 1.0, tp.ZeroField(), tp.ZeroField(), tp.ZeroField()))
    plan = tp.plan_boris(prob, tp.Boris(), dt=0.1, save_work=True)
    r = orc.boris_run(plan.desc, tp.ZeroField(), B, plan.u0)
    _, u = r.traj(0)
    # P_betatron = mu dB/dt . b with mu = |v_perp|^2 / (2 |B|), dB/dt = (0, 0, 1)
    assert np.all(u[:, 9] > 0.0)
