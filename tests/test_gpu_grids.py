"""GPU parity of the gridded fields off the trilinear fast path (orders 0 / 3,
rectilinear, spherical, 1-D / 2-D) and of tp_eval_points (get_fields /
get_work), against the CPU oracle on the same inputs.

Bars: Cartesian and rectilinear grids use +, -, *, / only and match the
oracle to 1e-13; spherical grids go through acos / atan2 / sincos, whose
CUDA and glibc results may differ in the last bit, and match to 1e-10 (the
bar of the multistep tests).  Jacobians (guiding centres, work rates) are
forward-mode derivatives on both sides.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_rows(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert a.shape == b.shape
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    a, b = np.where(na, 0.0, a), np.where(nb, 0.0, b)
    d = np.linalg.norm(a - b, axis=-1)
    r = np.linalg.norm(b, axis=-1)
    return float(np.max(np.where(r > 0, d / np.where(r > 0, r, 1.0), d))) if d.size else 0.0


def _turb(tp, n, order, bc, dtype=np.float32):
    dx = 1.0e5
    Ea, Ba, L = tp.workloads.turbulent_grid(n, dx, 5.0e-9, nmodes=8)
    x = np.arange(n) * dx
    B = tp.build_interpolator(Ba.astype(dtype), x, x, x, order, bc)
    E = tp.build_interpolator(Ea.astype(dtype), x, x, x, order, bc)
    return E, B, L


def _dipole_spherical(tp, order, nr=40, nth=37, nph=49):
    """The Earth dipole sampled on a spherical (r, theta, phi) grid, as
    (B_r, B_theta, B_phi) components."""
    r = np.geomspace(2.0 * tp.Re, 12.0 * tp.Re, nr) if order == 1 else np.linspace(2.0 * tp.Re, 12.0 * tp.Re, nr)
    th = np.linspace(0.0, math.pi, nth)
    ph = np.linspace(0.0, 2 * math.pi, nph)
    R, T, P = np.meshgrid(r, th, ph, indexing="ij")
    M = -tp.BMoment_Earth[2]
    k = tp.MU0_OVER_4PI * M / R ** 3
    A = np.zeros((3, nr, nth, nph))
    A[0] = -2.0 * k * np.cos(T)
    A[1] = -k * np.sin(T)
    return tp.build_interpolator(tp.StructuredGrid, A, r, th, ph, order)


def _grid_cases(tp):
    rng = np.random.default_rng(11)
    x = np.linspace(-1.0, 1.0, 9)
    xn = np.cumsum(rng.uniform(0.5, 1.5, 9))
    xn = 2 * (xn - xn[0]) / (xn[-1] - xn[0]) - 1.0
    A = rng.normal(size=(3, 9, 9, 9))
    cases = {
        "cubic_fill": tp.build_interpolator(A, x, x, x, 3),
        "cubic_periodic": tp.build_interpolator(A, x, x, x, 3, tp.PeriodicBC("exclusive")),
        "cubic_periodic_inclusive": tp.build_interpolator(A, x, x, x, 3, tp.PeriodicBC("inclusive")),
        "cubic_clamp": tp.build_interpolator(A.astype(np.float32), x, x, x, 3, tp.ClampExtrap()),
        "constant": tp.build_interpolator(A, x, x, x, 0, tp.ClampExtrap()),
        "rectilinear": tp.build_interpolator(tp.RectilinearGrid, A, xn, x, xn),
        "rectilinear_clamp": tp.build_interpolator(tp.RectilinearGrid, A, xn, x, xn, 1, tp.ClampExtrap()),
        "cartesian_2d": tp.build_interpolator(tp.CartesianGrid, A[:, :, :, 0], x, x, 3),
        "cartesian_1d": tp.build_interpolator(tp.CartesianGrid, A[:, :, 0, 0], x, 1, tp.FillExtrap(), dir=2),
    }
    r, th, ph = np.linspace(0.2, 1.5, 8), np.linspace(0, math.pi, 9), np.linspace(0, 2 * math.pi, 13)
    S = rng.normal(size=(3, 8, 9, 13))
    cases["spherical_linear"] = tp.build_interpolator(tp.StructuredGrid, S, r, th, ph, 1)
    cases["spherical_cubic"] = tp.build_interpolator(tp.StructuredGrid, S, r, th, ph, 3)
    cases["spherical_scalar"] = tp.build_interpolator(tp.StructuredGrid, S[0], np.geomspace(0.2, 1.5, 8), th, ph)
    return cases


@pytest.mark.parametrize("name", ["cubic_fill", "cubic_periodic", "cubic_periodic_inclusive", "cubic_clamp",
                                  "constant", "rectilinear", "rectilinear_clamp", "cartesian_2d", "cartesian_1d",
                                  "spherical_linear", "spherical_cubic", "spherical_scalar"])
def test_eval_points_fields_and_jacobian_work_match_oracle(tp, orc, name):
    F = _grid_cases(tp)[name]
    rng = np.random.default_rng(5)
    n = 4096
    pts = rng.uniform(-1.3, 1.3, (n, 3))   # inside and outside the grid
    u = np.concatenate([pts, rng.normal(size=(n, 3))], axis=1)
    t = np.zeros(n)
    ctx = tp.Context.get(0)
    E = tp.UniformField((0.3, -0.2, 0.5))
    out = ctx.eval_points(E, F, u, t, gc=False, want=3, q2m=1.0, m=2.0)
    ref, J = orc.field_eval(F, pts, jacobian=True)
    tol = 1e-10 if name.startswith("spherical") else 1e-13
    assert _rel_rows(out[:, 3:6], ref) <= tol
    assert np.all(out[:, 0:3] == np.array([0.3, -0.2, 0.5]))
    # work rates from the oracle's field and Jacobian (get_work_rates, equations.jl:394-441)
    W = np.full((n, 4), np.nan)
    for i in range(n):
        B, JB, v = ref[i], J[i], u[i, 3:6]
        if np.any(np.isnan(B)):
            continue
        Bm = math.sqrt((B[0] * B[0] + B[1] * B[1]) + B[2] * B[2])
        if Bm == 0:
            W[i] = 0.0
            continue
        b = B / Bm
        gB = JB.T @ b
        kap = (JB @ b + b * (-(gB @ b))) / Bm
        vp = v @ b
        vperp = v - vp * b
        mu = 2.0 * (vperp @ vperp) / (2 * Bm)
        Ev = np.array([0.3, -0.2, 0.5])
        W[i] = [2.0 * vp * (Ev @ b), (2.0 * vp * vp / Bm) * (np.cross(b, kap) @ Ev),
                (mu / Bm) * (np.cross(b, gB) @ Ev), 0.0]
    ok = ~np.isnan(W[:, 0])
    assert np.array_equal(ok, ~np.isnan(out[:, 6]))
    d = np.linalg.norm(out[ok, 6:10] - W[ok], axis=1)
    r = np.linalg.norm(W[ok], axis=1)
    assert np.all(d <= 1e-9 * r + 1e-12 * np.median(r))


@pytest.mark.parametrize("order", [0, 3])
def test_boris_cubic_and_constant_grid_fp64(tp, orc, order):
    E, B, L = _turb(tp, 24, order, tp.PeriodicBC("exclusive"), np.float64)
    rng = np.random.default_rng(2)
    n = 256
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(0.0, L, (3, n))
    u0[3:] = rng.normal(0.0, 1.5e5, (3, n))
    dt = tp.get_gyroperiod(5.0e-9) / 40
    prob = tp.TraceProblem(u0, (0.0, 800 * dt), tp.prepare(E, B))
    kw = dict(dt=dt, savestepinterval=200, save_fields=True)
    sols = tp.solve(prob, tp.Boris(), **kw)
    plan = tp.plan_boris(prob, tp.Boris(), **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
    assert np.array_equal(sols.nsaved, ref.nsaved)
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel_rows(sols.u_all[:, :3], ref.u[:, :3]) <= 1e-13
    assert _rel_rows(sols.u_all[:, 3:6], ref.u[:, 3:6]) <= 1e-13
    assert _rel_rows(sols.u_all[:, 9:12], ref.u[:, 9:12]) <= 1e-13
    # get_fields on the solution equals the saved columns
    Eg, Bg = tp.get_fields(sols)
    assert np.array_equal(Bg, sols.u_all[:, 9:12]) and np.array_equal(Eg, sols.u_all[:, 6:9])
    if order == 3:
        # this box is chaotic (float64 runs started 1e-7 apart separate by
        # O(L) within 800 steps): compare FP32C over 100 steps, where such
        # runs stay within a median of ~1e-6 L
        short = tp.TraceProblem(u0, (0.0, 100 * dt), tp.prepare(E, B))
        s32 = tp.solve(short, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=dt, savestepinterval=100)
        p64 = tp.plan_boris(short, tp.Boris(), dt=dt, savestepinterval=100)
        r64 = orc.boris_run(p64.desc, p64.E, p64.B, p64.u0)
        d = np.abs(s32.final_states()[:, :3] - r64.final_states()[:, :3]).max(axis=1)
        assert np.median(d) <= 1e-5 * L


def test_boris_rectilinear_and_2d_grid_fp64(tp, orc):
    rng = np.random.default_rng(4)
    x = np.cumsum(rng.uniform(0.5, 1.5, 33)) * 1.0e5
    x -= x[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    L = x[-1]
    Ba = np.zeros((3, 33, 33, 33))
    Ba[2] = 5.0e-9 * (1.0 + 0.2 * np.sin(2 * math.pi * X / L))
    Ba[0] = 1.0e-9 * np.cos(2 * math.pi * Y / L)
    B = tp.build_interpolator(tp.RectilinearGrid, Ba, x, x, x, 1, tp.ClampExtrap())
    B2 = tp.build_interpolator(tp.CartesianGrid, Ba[:, :, :, 0], np.linspace(0, L, 33), np.linspace(0, L, 33),
                               1, tp.ClampExtrap())
    n = 256
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(0.2 * L, 0.8 * L, (3, n))
    u0[3:] = rng.normal(0.0, 1.0e5, (3, n))
    dt = tp.get_gyroperiod(5.0e-9) / 40
    for F in (B, B2):
        prob = tp.TraceProblem(u0, (0.0, 600 * dt), tp.prepare(tp.ZeroField(), F))
        kw = dict(dt=dt, savestepinterval=150, save_work=True)
        sols = tp.solve(prob, tp.Boris(), **kw)
        plan = tp.plan_boris(prob, tp.Boris(), **kw)
        ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
        assert np.array_equal(sols.nsaved, ref.nsaved)
        assert _rel_rows(sols.u_all[:, :3], ref.u[:, :3]) <= 1e-13
        assert _rel_rows(sols.u_all[:, 3:6], ref.u[:, 3:6]) <= 1e-13
        assert np.array_equal(tp.get_work(sols), sols.u_all[:, 6:10])


@pytest.mark.parametrize("order", [1, 3])
def test_dipole_on_spherical_grid_boris_and_gc(tp, orc, order):
    B = _dipole_spherical(tp, order)
    # full orbit: 100 keV protons at 4 - 6 R_E
    rng = np.random.default_rng(8)
    n = 128
    r = rng.uniform(4.0, 6.0, n) * tp.Re
    th = rng.uniform(0.35 * math.pi, 0.65 * math.pi, n)
    ph = rng.uniform(0, 2 * math.pi, n)
    x = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)])
    vmag = tp.energy2velocity(1.0e5)
    vd = rng.normal(size=(3, n))
    vd /= np.linalg.norm(vd, axis=0)
    u0 = np.concatenate([x, vmag * vd])
    dt = 0.01
    prob = tp.TraceProblem(u0, (0.0, 400 * dt), tp.prepare(tp.ZeroField(), B, species=tp.Proton))
    kw = dict(dt=dt, savestepinterval=100)
    sols = tp.solve(prob, tp.Boris(), **kw)
    plan = tp.plan_boris(prob, tp.Boris(), **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
    assert np.array_equal(sols.nsaved, ref.nsaved)
    assert _rel_rows(sols.u_all[:, :3], ref.u[:, :3]) <= 1e-10
    # the gridded dipole stays close to the analytic one
    an = tp.solve(tp.TraceProblem(u0, (0.0, 400 * dt),
                                  tp.prepare(tp.ZeroField(), tp.DipoleField(tp.BMoment_Earth), species=tp.Proton)),
                  tp.Boris(), **kw)
    dpos = np.linalg.norm(an.final_states()[:, :3] - sols.final_states()[:, :3], axis=1)
    assert np.median(dpos / np.linalg.norm(an.final_states()[:, :3], axis=1)) <= 1e-2
    # guiding centre RK4 (needs the grid's Jacobian)
    y0, mu = orc.gc_prepare(tp.ZeroField(), B, u0.T.copy(), tp.qi, tp.mi)
    gprob = tp.TraceGCProblem(y0.T.copy(), (0.0, 20.0), (tp.qi, tp.qi / tp.mi, mu, tp.ZeroField(), B))
    gkw = dict(dt=0.05, alg="rk4", savestepinterval=100, save_work=True)
    gs = tp.solve(gprob, **gkw)
    gp = tp.plan_gc(gprob, **gkw)
    gr = orc.gc_run(gp.desc, gp.E, gp.B, gp.y0, gp.q_i, gp.q2m_i, gp.mu_i)
    assert np.array_equal(gs.nsaved, gr.nsaved)
    assert _rel_rows(gs.u_all[:, :3], gr.u[:, :3]) <= 1e-10
    # E = 0 and a static B: no work wherever the guiding centre is on the grid
    # (mirror points below 2 R_E leave it and read NaN, on both sides)
    w = gs.u_all[:, 4:8]
    assert np.array_equal(np.isnan(w), np.isnan(gr.u[:, 4:8]))
    assert np.all(w[np.isfinite(w)] == 0.0)


def test_gc_cubic_grid_rk45(tp, orc):
    E, B, L = _turb(tp, 24, 3, tp.PeriodicBC("exclusive"), np.float64)
    rng = np.random.default_rng(9)
    n = 128
    xv = np.concatenate([rng.uniform(0, L, (n, 3)), rng.normal(0, 1.0e5, (n, 3))], axis=1)
    y0, mu = orc.gc_prepare(E, B, xv, tp.qi, tp.mi)
    prob = tp.TraceGCProblem(y0.T.copy(), (0.0, 50.0), (tp.qi, tp.qi / tp.mi, mu, E, B))
    for alg in ("rk4", "rk45"):
        kw = dict(dt=0.05, alg=alg, savestepinterval=100, maxiters=4000)
        s = tp.solve(prob, **kw)
        p = tp.plan_gc(prob, **kw)
        r = orc.gc_run(p.desc, p.E, p.B, p.y0, p.q_i, p.q2m_i, p.mu_i)
        assert np.array_equal(s.nsaved, r.nsaved)
        assert _rel_rows(s.u_all[:, :3], r.u[:, :3]) <= (1e-12 if alg == "rk4" else 1e-9)


# ------------------------------------------------------------------ time series (LazyTimeInterpolator)
def _series(tp, nsnap=5, n=16, order=1):
    """Snapshots of the turbulent box whose fluctuation amplitude grows in time."""
    dx = 1.0e5
    Ea, Ba, L = tp.workloads.turbulent_grid(n, dx, 5.0e-9, nmodes=8)
    x = np.arange(n) * dx
    B0 = np.zeros_like(Ba)
    B0[2] = 5.0e-9
    times = np.linspace(0.0, 40.0, nsnap)

    def loader(i):
        a = (i - 1) / max(nsnap - 1, 1)
        return tp.build_interpolator((B0 + a * (Ba - B0)).astype(np.float64), x, x, x, order,
                                     tp.PeriodicBC("exclusive"))

    return tp.LazyTimeInterpolator(times, loader), L


def test_series_eval_points_and_work_match_oracle(tp, orc):
    B, L = _series(tp)
    rng = np.random.default_rng(1)
    n = 4096
    u = np.concatenate([rng.uniform(0, L, (n, 3)), rng.normal(0, 1e5, (n, 3))], axis=1)
    t = rng.uniform(-5.0, 45.0, n)   # before, inside and after the snapshot times
    ctx = tp.Context.get(0)
    E = tp.UniformField((0.0, 1.0e-4, 0.0))
    out = ctx.eval_points(E, B, u, t, gc=False, want=3, q2m=tp.qi / tp.mi, m=tp.mi)
    for k in range(0, n, 97):
        ref, J = orc.field_eval(B, u[k, :3], t[k], jacobian=True)
        assert _rel_rows(out[k:k + 1, 3:6], ref) <= 1e-13
    # the betatron term follows dB/dt of the series: nonzero inside, zero outside
    inside = (t > 0.0) & (t < 40.0)
    assert np.any(out[inside, 9] != 0.0) and np.all(out[~inside, 9] == 0.0)


def test_series_boris_and_gc_match_oracle(tp, orc):
    B, L = _series(tp)
    rng = np.random.default_rng(6)
    n = 256
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(0.0, L, (3, n))
    u0[3:] = rng.normal(0.0, 1.0e5, (3, n))
    dt = tp.get_gyroperiod(5.0e-9) / 40
    prob = tp.TraceProblem(u0, (0.0, 120 * dt), tp.prepare(tp.ZeroField(), B))
    kw = dict(dt=dt, savestepinterval=30, save_work=True)
    sols = tp.solve(prob, tp.Boris(), **kw)
    plan = tp.plan_boris(prob, tp.Boris(), **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
    assert np.array_equal(sols.nsaved, ref.nsaved)
    assert _rel_rows(sols.u_all[:, :3], ref.u[:, :3]) <= 1e-13
    assert _rel_rows(sols.u_all[:, 3:6], ref.u[:, 3:6]) <= 1e-13
    d = np.linalg.norm(sols.u_all[:, 6:10] - ref.u[:, 6:10], axis=1)
    assert np.all(d <= 1e-12 * np.linalg.norm(ref.u[:, 6:10], axis=1) + 1e-30)
    s32 = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=dt, savestepinterval=30)
    e = np.linalg.norm(s32.final_states()[:, :3] - ref.final_states()[:, :3], axis=1)
    assert np.median(e) <= 1e-5 * L
    xv = np.concatenate([u0[:3].T, u0[3:].T], axis=1)
    y0, mu = orc.gc_prepare(tp.ZeroField(), B, xv, tp.qi, tp.mi)
    gprob = tp.TraceGCProblem(y0.T.copy(), (0.0, 30.0), (tp.qi, tp.qi / tp.mi, mu, tp.ZeroField(), B))
    gkw = dict(dt=0.05, alg="rk4", savestepinterval=100)
    gs = tp.solve(gprob, **gkw)
    gp = tp.plan_gc(gprob, **gkw)
    gr = orc.gc_run(gp.desc, gp.E, gp.B, gp.y0, gp.q_i, gp.q2m_i, gp.mu_i)
    assert np.array_equal(gs.nsaved, gr.nsaved)
    assert _rel_rows(gs.u_all[:, :3], gr.u[:, :3]) <= 1e-12


@pytest.mark.parametrize("alg", ["boris", "multistep"])
def test_cubic_grid_fp32c_warp_cooperative_kernel(tp, orc, alg):
    """E and B on one periodic cubic grid take the warp-cooperative FP32C
    kernel (one particle's 64-node stencil gathered by the whole warp).  Uneven
    lifetimes (per-particle dt, a box that stops some orbits), a partial last
    warp and saved fields, against the float64 oracle over ~1.5 gyroperiods."""
    E, B, L = _turb(tp, 20, 3, tp.PeriodicBC("exclusive"))
    rng = np.random.default_rng(11)
    n = 1000
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(0.3 * L, 0.7 * L, (3, n))
    u0[3:] = rng.normal(0.0, 1.0e5, (3, n))
    T = tp.get_gyroperiod(5.0e-9)
    dt = (T / 40) * rng.uniform(0.9, 1.1, n)
    a = tp.Boris() if alg == "boris" else tp.MultistepBoris4(2)
    prob = tp.TraceProblem(u0, (0.0, 1.5 * T), tp.prepare(E, B))
    # orbits stream along B (z) and drift across x and y by about L within the
    # span: a box of [-L/2, 3L/2] in y stops about a fifth of them (oracle)
    box = tp.TerminateBox((-np.inf, -0.5 * L, -np.inf), (np.inf, 1.5 * L, np.inf))
    kw = dict(dt=dt, savestepinterval=20, save_fields=True, isoutside=box)
    s32 = tp.solve(prob, a, tp.EnsembleB200(precision="fp32c"), **kw)
    plan = tp.plan_boris(prob, a, **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    assert np.array_equal(s32.nsaved, ref.nsaved) and np.array_equal(s32.retcodes, ref.retcode)
    assert 0 < np.sum(ref.retcode == 2) < n  # some orbits stop at the box, some do not
    assert np.array_equal(s32.t_all, ref.t)
    d = np.abs(s32.u_all[:, :3] - ref.u[:, :3]).max(axis=1)
    assert np.max(d) <= 1e-5 * L
    assert _rel_rows(s32.u_all[:, 3:6], ref.u[:, 3:6]) <= 1e-4
    # the saved fields are the kernel's float evaluation at the saved positions:
    # against the float64 evaluation at those same positions
    Eg, Bg = tp.get_fields(s32)
    assert _rel_rows(s32.u_all[:, 9:12], Bg) <= 1e-5 and _rel_rows(s32.u_all[:, 6:9], Eg) <= 1e-5
