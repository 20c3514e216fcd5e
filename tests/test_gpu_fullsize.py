"""Parity at the full sizes of the benchmark workloads (configs 2-5).

The oracle cannot run a million particles for 1e4 steps in a test, but
particles are independent: for any subset of a full-size ensemble, the
device's results must equal the oracle's run of that subset alone.  Each test
runs one workload at full size on the device (through the C ABI), draws a
seeded subset of 256 particles, and checks:

  * FP64 runs: the subset's save counts, return codes, step counts and saved
    states equal the oracle's.  Bars as in the small-size parity tests:
    states <= 1e-13 relative for +-*/sqrt arithmetic, <= 1e-10 where CUDA's
    and glibc's atan / sincos / pow may differ in the last bit (1e-9 for the
    multistep push over 1e4 steps).
  * FP32C runs: the subset's trajectories inside the full run are bitwise
    equal to a device run of the subset alone (no cross-particle effects at
    full occupancy), and the final-position error against the float64 oracle
    stays within the chaotic separation of two float64 runs started 1 ulp
    apart (the stated FP32C error).
  * The adjoint: forward states and dL/du0 of the subset are bitwise equal to
    those of a run of the subset alone; node gradients are linear in the
    cotangent, and their sum is the uniform-offset parameter gradient.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSUB = 256


def _subset(n, seed, k=NSUB):
    return np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False))


def _rows(sol, idx):
    """Packed (t, u) rows of trajectories idx, in order."""
    o = sol.offsets
    sel = np.concatenate([np.arange(o[i], o[i + 1]) for i in idx])
    return sol.t_all[sel], sol.u_all[sel]


def _rel_rows(a, b):
    """max over rows of |a - b| / |b| per 3-vector block (positions, velocities)."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert a.shape == b.shape
    assert np.array_equal(np.isnan(a), np.isnan(b))
    a, b = np.where(np.isnan(a), 0.0, a), np.where(np.isnan(b), 0.0, b)
    worst = 0.0
    for lo in range(0, a.shape[1], 3):
        hi = min(lo + 3, a.shape[1])
        d = np.linalg.norm(a[:, lo:hi] - b[:, lo:hi], axis=1)
        r = np.linalg.norm(b[:, lo:hi], axis=1)
        worst = max(worst, float(np.max(d / np.where(r > 0, r, 1.0))))
    return worst


def _check_subset(sol, idx, ref, tol):
    assert np.array_equal(sol.nsaved[idx], ref.nsaved)
    assert np.array_equal(sol.retcodes[idx], ref.retcode)
    assert np.array_equal(sol.nsteps[idx], ref.nsteps)
    t, u = _rows(sol, idx)
    assert _rel_rows(t[:, None], ref.t[:, None]) <= tol
    assert _rel_rows(u, ref.u) <= tol


def _same_trajectories(full, idx, sub):
    assert np.array_equal(full.nsaved[idx], sub.nsaved)
    assert np.array_equal(full.retcodes[idx], sub.retcodes)
    assert np.array_equal(full.nsteps[idx], sub.nsteps)
    t, u = _rows(full, idx)
    assert np.array_equal(t, sub.t_all)
    assert np.array_equal(u, sub.u_all)


def _final_pos_err(a, b):
    return np.linalg.norm(a[:, :3] - b[:, :3], axis=1) / np.linalg.norm(b[:, :3], axis=1)


def test_config2_full_size(tp, orc):
    """1e6 protons x 1e4 Boris steps in the 128^3 turbulent field, saves every 1000."""
    w = tp.workloads.config2()
    assert w.n == 1_000_000 and w.nt == 10_000
    kw = dict(dt=w.dt, savestepinterval=w.savestepinterval)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    idx = _subset(w.n, 21)
    sub = tp.TraceProblem(w.u0[:, idx].copy(), w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(sub, tp.Boris(), tp.EnsembleB200(precision="fp64"), **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)

    s64 = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp64"), **kw)
    assert int(s64.nsteps.sum()) == w.n * w.nt
    _check_subset(s64, idx, ref, 1e-13)
    del s64

    s32 = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), **kw)
    _same_trajectories(s32, idx, tp.solve(sub, tp.Boris(), tp.EnsembleB200(precision="fp32c"), **kw))
    # stated error: FP32C against float64 within the separation of float64
    # runs started one ulp apart (the field is chaotic over 1e4 steps)
    u1 = plan.u0.copy()
    u1[:, 0] = np.nextafter(u1[:, 0], np.inf)
    ref1 = orc.boris_run(plan.desc, plan.E, plan.B, u1)
    fin = s32.final_states()[idx]
    e32 = np.median(_final_pos_err(fin, ref.final_states()))
    e64 = np.median(_final_pos_err(ref1.final_states(), ref.final_states()))
    assert e32 <= 3.0 * e64 + 1e-6


def test_config3_full_size(tp, orc):
    """1e6 protons in the Earth dipole: AdaptiveBoris(0.1) (cap 1e4 steps) and MultistepBoris4(2)."""
    w = tp.workloads.config3()
    assert w.n == 1_000_000
    idx = _subset(w.n, 31)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    sub = tp.TraceProblem(w.u0[:, idx].copy(), w.tspan, tp.prepare(w.E, w.B, species=w.species))

    kw = dict(tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside, step_cap=w.nt)
    subkw = dict(kw, tend=w.tend[idx])
    sa = tp.solve(prob, tp.AdaptiveBoris(0.1), tp.EnsembleB200(precision="fp64"), **kw)
    plan = tp.plan_boris(sub, tp.AdaptiveBoris(0.1), tp.EnsembleB200(precision="fp64"), **subkw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    _check_subset(sa, idx, ref, 1e-13)   # identical step decisions
    t, _ = _rows(sa, idx)
    assert np.array_equal(t, ref.t)
    del sa

    kw = dict(dt=w.dt, tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    subkw = dict(kw, dt=w.dt[idx], tend=w.tend[idx])
    sm = tp.solve(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp64"), **kw)
    plan = tp.plan_boris(sub, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp64"), **subkw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    # atan and sincos are the portable routines the oracle shares, so every
    # orbit -- the chaotic 10 MeV tail included -- takes the same steps and
    # the same saves as the oracle, to the last bit or nearly (1e-13)
    _check_subset(sm, idx, ref, 1e-13)
    t, _ = _rows(sm, idx)
    assert np.array_equal(t, ref.t)
    del sm
    s32 = tp.solve(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp32c"), **kw)
    _same_trajectories(s32, idx, tp.solve(sub, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp32c"),
                                          **subkw))


@pytest.mark.parametrize("alg", ["rk4", "rk45"])
def test_config4_full_size(tp, orc, alg):
    """2^20 guiding centres in the dipole over 5 bounce periods."""
    w = tp.workloads.config4()
    assert w.n == 1 << 20
    idx = _subset(w.n, 41)
    kw = dict(tend=5 * w.tau_b, alg=alg, savestepinterval=100_000, save_everystep=False, maxiters=1_000_000)
    kw.update(dict(dt=w.tau_b / 200) if alg == "rk4" else dict(abstol=1e-9, reltol=1e-6))
    prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
    sol = tp.solve(prob, tp.EnsembleB200(precision="fp64"), **kw)
    sub = tp.TraceGCProblem(w.y0[:, idx].copy(), (0.0, 1.0), (w.q[idx], w.q2m[idx], w.mu[idx], w.E, w.B))
    subkw = dict(kw, tend=kw["tend"][idx])
    if alg == "rk4":
        subkw["dt"] = kw["dt"][idx]
    plan = tp.plan_gc(sub, **subkw)
    ref = orc.gc_run(plan.desc, plan.E, plan.B, plan.y0, plan.q_i, plan.q2m_i, plan.mu_i,
                     dt_i=plan.dt_i, tend_i=plan.tend_i)
    _check_subset(sol, idx, ref, 1e-12 if alg == "rk4" else 1e-10)
    s32 = tp.solve(prob, tp.EnsembleB200(precision="fp32"), **kw)
    _same_trajectories(s32, idx, tp.solve(sub, tp.EnsembleB200(precision="fp32"), **subkw))


def test_config5_adjoint_full_size(tp):
    """2^18 protons x 4096 steps, checkpoints every 64: the adjoint at full size."""
    w = tp.workloads.config5()
    assert w.n == 1 << 18 and w.nt == 4096
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    uf, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=64)
    rng = np.random.default_rng(51)
    c1 = rng.normal(size=(w.n, 6)) * np.array([1e-7] * 3 + [1e-6] * 3)
    c2 = rng.normal(size=(w.n, 6)) * np.array([1e-7] * 3 + [1e-6] * 3)
    g1 = tape.backward(c1)
    g2 = tape.backward(c2)
    g12 = tape.backward(c1 + c2)

    idx = _subset(w.n, 52)
    sub = tp.TraceProblem(w.u0[:, idx].copy(), w.tspan, tp.prepare(w.E, w.B, species=w.species))
    ufs, tsub = tp.adjoint_solve(sub, dt=w.dt, checkpoint_every=64)
    assert np.array_equal(uf[idx], ufs)
    assert np.array_equal(g1.u0[idx], tsub.backward(c1[idx], fields=False).u0)

    for a, b, ab in ((g1.E, g2.E, g12.E), (g1.B, g2.B, g12.B)):
        a, b, ab = (np.asarray(x, np.float64) for x in (a, b, ab))
        scale = np.abs(ab).max()
        assert scale > 0.0 and np.all(np.isfinite(ab))
        assert np.allclose(a + b, ab, rtol=1e-3, atol=1e-5 * scale)
    # the uniform-offset parameter gradients are the node-gradient sums
    for g in (g1, g12):
        for k, table in ((0, g.E), (3, g.B)):
            a = np.asarray(table, np.float64).reshape(3, -1)
            s = a.sum(axis=1)
            assert np.all(np.abs(g.param[k:k + 3] - s) <= 1e-12 * np.abs(a).sum(axis=1))


def test_config4_get_work_is_one_launch(tp):
    """get_work / get_fields of 2^20 guiding centres that carry their own q, q/m
    and mu: one tp_eval_points_params call for the whole ensemble, equal to the
    save_work columns the solve wrote (same kernel code, same states)."""
    w = tp.workloads.config4()
    prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
    sols = tp.solve(prob, tp.EnsembleB200(), alg="rk4", dt=w.tau_b / 200, tend=0.05 * w.tau_b, savestepinterval=5,
                    save_work=True)
    ctx = tp.Context.get(0)
    calls = []
    orig = ctx.eval_points

    def counted(*a, **k):
        calls.append(1)
        return orig(*a, **k)

    ctx.eval_points = counted
    try:
        work = tp.get_work(sols)
    finally:
        del ctx.eval_points
    assert len(calls) == 1
    assert work.shape == (sols.t_all.size, 4)
    assert np.array_equal(work, sols.u_all[:, 4:8])
