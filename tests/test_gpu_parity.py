"""GPU parity: the CUDA library against the CPU oracle on the same seeded inputs.

Bars (per the reference's own kernel-vs-native test, test_boris_kernel.jl:92):
  * FP64 Boris / adaptive Boris / GC, +-*/sqrt-only arithmetic: identical to
    the oracle (both follow the reference's operation order, no contraction);
    asserted as relative error <= 1e-13.
  * FP64 MultistepBoris (CUDA vs glibc atan/sincos differ in the last bit):
    relative error <= 1e-10 after the stated steps.
  * FP32C: relative position error <= 1e-5 against the float64 oracle on
    non-chaotic (uniform / dipole) cases, stated for gridded turbulence.
All calls go through the C ABI (libtpb200.so) via the package's solve().
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import julia_isapprox

pytestmark = pytest.mark.gpu


def _rel(a, b, blocks=None):
    """Largest relative difference of saved states, per vector: |dx|/|x| for the
    position (or guiding-centre position) and |dv|/|v| for the velocity block
    (v_par for guiding centres; saved fields compared as one block each; work
    rates as one 4-vector).  `blocks` overrides the column grouping.
    NaN entries must coincide."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    if a.shape != b.shape:
        return np.inf
    if a.size == 0:
        return 0.0
    if a.ndim == 1:
        a, b = a[:, None], b[:, None]
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    if not np.array_equal(nan_a, nan_b):
        return np.inf
    a = np.where(nan_a, 0.0, a)
    b = np.where(nan_b, 0.0, b)
    W = a.shape[1]
    if blocks is None:
        blocks = {1: [(0, 1)], 4: [(0, 3), (3, 4)], 6: [(0, 3), (3, 6)],
                  10: [(0, 3), (3, 4), (4, 7), (7, 10)], 12: [(0, 3), (3, 6), (6, 9), (9, 12)],
                  14: [(0, 3), (3, 4), (4, 7), (7, 10), (10, 14)],
                  16: [(0, 3), (3, 6), (6, 9), (9, 12), (12, 16)]}.get(W, [(c, c + 1) for c in range(W)])
    worst = 0.0
    for lo, hi in blocks:
        d = np.linalg.norm(a[:, lo:hi] - b[:, lo:hi], axis=1)
        r = np.linalg.norm(b[:, lo:hi], axis=1)
        ok = r > 0
        if np.any(d[~ok] > 0):
            worst = max(worst, float(np.max(d[~ok])))  # absolute where the reference is 0
        if np.any(ok):
            worst = max(worst, float(np.max(d[ok] / r[ok])))
    return worst


def _pos_rel(gpu_u, ref_u):
    """max over saves of |x_gpu - x_ref| / |x_ref| (positions only)."""
    d = np.linalg.norm(gpu_u[:, :3] - ref_u[:, :3], axis=1)
    r = np.linalg.norm(ref_u[:, :3], axis=1)
    return float(np.max(d / np.maximum(r, 1e-300)))


def _both(tp, orc, prob, alg, ens=None, **kw):
    ens = ens or tp.EnsembleB200()
    sols = tp.solve(prob, alg, ens, **kw)
    plan = tp.plan_boris(prob, alg, ens, **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    return sols, ref


def _check_same_layout(sols, ref):
    assert np.array_equal(sols.nsaved, ref.nsaved)
    assert np.array_equal(sols.retcodes, ref.retcode)
    assert np.array_equal(sols.nsteps, ref.nsteps)


# ------------------------------------------------------------------ config 1 (CPU-runnable)
def test_config1_plain_boris_fp64_matches_oracle(tp, orc):
    w = tp.workloads.config1()
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=tp.Proton))
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=w.dt, savestepinterval=w.savestepinterval)
    _check_same_layout(sols, ref)
    assert sols.nsaved[0] == 101
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel(sols.u_all, ref.u) <= 1e-13
    # |v| conserved under pure-B rotation to float64 round-off
    v0 = np.linalg.norm(w.u0[3:6].T, axis=1)
    vend = np.linalg.norm(sols.final_states()[:, 3:6], axis=1)
    assert np.max(np.abs(vend - v0) / v0) < 1e-12


def test_reference_boris_kats_on_gpu(tp):
    # test_boris.jl:40-61 through the B200 path
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param)
    sol = tp.solve(prob, tp.Boris(), dt=3.0e-11, savestepinterval=10).u[0]
    assert julia_isapprox(sol.u[-1], [-0.00010199137926394769, 3.46340469171306e-5, 0.0,
                                      -60893.043824907196, -79322.36263335795, 0.0])
    assert julia_isapprox(sol(1.5e-8), [-3.8587882024745045e-5, 5.3855907133664956e-5, 0.0,
                                        -94689.58829601014, 32154.033469101283, 0.0])
    assert sol.retcode == "Success" and len(sol.t) == 101

    def pf(prob, ctx):
        u = list(prob.u0)
        u[4] = ctx.sim_id * 1.0e5
        return tp.remake(prob, u0=u)

    prob = tp.TraceProblem([0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param, prob_func=pf)
    sols = tp.solve(prob, tp.Boris(), tp.EnsembleB200(), dt=3.0e-11, savestepinterval=1000, trajectories=4)
    assert julia_isapprox(sum(s.u[-1][3] for s in sols.u), -608930.4382490724)


@pytest.mark.parametrize("flags,n_expected", [
    (dict(savestepinterval=10), 101),
    (dict(savestepinterval=10, save_everystep=False, save_start=False, save_end=True), 1),
    (dict(savestepinterval=10, save_everystep=False, save_start=True, save_end=True), 2),
    (dict(savestepinterval=10, save_everystep=False, save_start=True, save_end=False), 1),
    (dict(savestepinterval=10, save_everystep=True, save_start=False, save_end=False), 99),
    (dict(savestepinterval=3, save_everystep=True, save_start=True, save_end=True), 335),
])
def test_saving_flags_gpu(tp, orc, flags, n_expected):
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3.0e-8), param)
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=3.0e-11, **flags)
    _check_same_layout(sols, ref)
    assert sols.nsaved[0] == n_expected
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel(sols.u_all, ref.u) <= 1e-13


def test_save_fields_gpu(tp, orc):
    w = tp.workloads.config1(64)
    prob = tp.TraceProblem(w.u0, (0.0, 500 * w.dt), tp.prepare(w.E, w.B))
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=w.dt, savestepinterval=50, save_fields=True)
    assert sols.u_all.shape[1] == 12
    assert _rel(sols.u_all, ref.u) <= 1e-13


# ------------------------------------------------------------------ work rates at save points
_WORK10 = [(0, 3), (3, 6), (6, 10)]   # full orbit: x, v, (P_par, P_fermi, P_grad, P_betatron)


def _work_problem(tp, n=64, betatron=False):
    """test_boris.jl:374-466 fields (constant_E and gradient_B, or the linear
    betatron B), electrons with spread initial velocities."""
    rng = np.random.default_rng(5)
    u0 = np.zeros((6, n))
    u0[:3] = rng.uniform(-1e-4, 1e-4, (3, n))
    u0[3:] = rng.normal(0.0, 1.0e5, (3, n))
    if betatron:
        E, B = tp.ZeroField(), tp.AffineField((0.0, 0.0, 0.01), rate=(0.0, 0.0, 1.0e5))
    else:
        E = tp.UniformField((0.0, 1.0e5, 0.0))
        B = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    return tp.TraceProblem(u0, (0.0, 1.0e-9), tp.prepare(E, B, species=tp.Electron))


@pytest.mark.parametrize("alg", ["boris", "ms2n2", "ms4n2", "adaptive"])
def test_save_work_matches_oracle(tp, orc, alg):
    prob = _work_problem(tp)
    a = {"boris": tp.Boris(), "ms2n2": tp.MultistepBoris(2, 2), "ms4n2": tp.MultistepBoris(4, 2),
         "adaptive": tp.AdaptiveBoris(0.1)}[alg]
    kw = dict(savestepinterval=1, save_work=True) if alg == "adaptive" else \
        dict(dt=1.0e-11, savestepinterval=1, save_work=True)
    sols, ref = _both(tp, orc, prob, a, **kw)
    _check_same_layout(sols, ref)
    assert sols.u_all.shape[1] == 10
    tol = 1e-10 if alg.startswith("ms") else 1e-13   # CUDA vs glibc atan / sincos
    assert _rel(sols.u_all, ref.u, _WORK10) <= tol
    first = sols.u[0].u[0]
    assert abs(first[6]) <= 1e-10 * 1e5 and abs(first[8]) > 0.0
    # both flags: 16 columns, work after E and B, equal to the work-only run
    s16, r16 = _both(tp, orc, prob, a, save_fields=True, **kw)
    assert s16.u_all.shape[1] == 16
    assert _rel(s16.u_all, r16.u) <= tol
    assert np.array_equal(s16.u_all[:, 12:16], sols.u_all[:, 6:10])


def test_save_work_betatron_gpu(tp, orc):
    prob = _work_problem(tp, betatron=True)
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=1.0e-11, savestepinterval=10, save_work=True)
    _check_same_layout(sols, ref)
    assert _rel(sols.u_all, ref.u, _WORK10) <= 1e-13
    assert np.all(sols.u_all[:, 9] > 0.0)   # P_betatron = mu dB/dt . b > 0


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_save_work_dipole_and_grid(tp, orc, precision):
    w, prob, keep = _regular_dipole(tp, 128, 1000, 250)
    w.dt, w.tend = w.dt[keep], w.tend[keep]
    # a dawn-dusk electric field makes all three electric work terms nonzero
    prob = tp.TraceProblem(prob.u0, prob.tspan, tp.prepare(tp.UniformField((0.0, 1.0e-3, 0.0)), w.B,
                                                           species=tp.Proton))
    ens = tp.EnsembleB200(precision=precision)
    kw = dict(dt=w.dt, tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside, save_work=True,
              save_fields=True)
    sols = tp.solve(prob, tp.Boris(), ens, **kw)
    plan = tp.plan_boris(prob, tp.Boris(), **kw)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    _check_same_layout(sols, ref)
    assert np.all(np.abs(ref.u[:, 12:15]).max(axis=0) > 0.0)
    if precision == "fp64":
        assert _rel(sols.u_all, ref.u) <= 1e-13
    else:
        # saved fields come from the float32 evaluation, work rates from float64
        # arithmetic on the compensated state: both follow the state's error
        assert _rel(sols.u_all[:, 12:16], ref.u[:, 12:16], [(0, 4)]) <= 1e-3
    gprob, dt, ssi = _small_grid_workload(tp, n=256, nt=1000, ssi=250)
    sols, ref = _both(tp, orc, gprob, tp.Boris(), dt=dt, savestepinterval=ssi, save_work=True)
    _check_same_layout(sols, ref)
    assert _rel(sols.u_all, ref.u, _WORK10) <= 1e-13


def test_argument_errors_gpu(tp):
    E = tp.UniformField((0.0, 1.0e5, 0.0))
    B = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 1.0e5, 0.0, 0.0], (0.0, 1.0e-9), tp.prepare(E, B, species=tp.Electron))
    with pytest.raises(tp.ArgumentError):
        tp.solve(prob, tp.Boris(), dt=1.0e-11, maxiters=50)
    with pytest.raises(tp.ArgumentError):
        tp.solve(prob, tp.Boris(), dt=np.finfo(float).eps)


# ------------------------------------------------------------------ multistep / dipole
def _regular_dipole(tp, n, nt, ssi):
    """Dipole-ensemble particles below 1 MeV: adiabatic, regular orbits."""
    w = tp.workloads.config3(4 * n, nt=nt, ssi=ssi)
    keep = np.flatnonzero(w.extra["Ek_eV"] < 1.0e6)[:n]
    return w, tp.TraceProblem(w.u0[:, keep].copy(), w.tspan, tp.prepare(w.E, w.B, species=tp.Proton)), keep


def _dipole_sample(tp, n, nt, ssi):
    """The first n particles of the dipole ensemble (10 keV - 10 MeV, L 3-7):
    adiabatic orbits and the chaotic, non-adiabatic high-energy tail alike."""
    w = tp.workloads.config3(n, nt=nt, ssi=ssi)
    return w, tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=tp.Proton))


@pytest.mark.parametrize("N,n", [(2, 1), (2, 2), (4, 2), (6, 2), (4, 1)])
def test_multistep_dipole_fp64(tp, orc, N, n):
    # atan / sincos of multistep_boris.jl:110-119 are the portable routines the
    # oracle shares, so even chaotic orbits agree to the last bits
    w, prob = _dipole_sample(tp, 256, 2000, 500)
    sols, ref = _both(tp, orc, prob, tp.MultistepBoris(N, n), dt=w.dt, tend=w.tend,
                      savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    _check_same_layout(sols, ref)
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel(sols.u_all, ref.u) <= 1e-13


def test_multistep_exb_and_gyration_gpu(tp):
    # test_boris.jl:95-210 through the B200 path
    param = (1.0, 1.0, tp.UniformField((0.0, 1.0, 0.0)), tp.UniformField((0.0, 0.0, 1.0)), tp.ZeroField())
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0.0, 10.0), param)
    for alg in (tp.Boris(), tp.MultistepBoris(2, 2), tp.MultistepBoris(4, 2), tp.MultistepBoris(6, 2)):
        end = tp.solve(prob, alg, dt=0.1).u[0].u[-1]
        assert abs(end[0] - 10.0) <= 1e-6 and abs(end[3] - 1.0) <= 1e-6
    param = (1.0, 1.0, tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0)), tp.ZeroField())
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 1.0, 0.0, 0.0], (0.0, 2 * math.pi), param)
    for alg in (tp.Boris(), tp.MultistepBoris(2, 4), tp.MultistepBoris(4, 4), tp.MultistepBoris(6, 4)):
        end = tp.solve(prob, alg, dt=0.1).u[0].u[-1]
        assert math.hypot(*end[:3]) < 0.02 and abs(math.hypot(*end[3:6]) - 1.0) <= 2.0e-3


# ------------------------------------------------------------------ adaptive
@pytest.mark.parametrize("alg", ["adaptive", "adaptive_ms4"])
def test_adaptive_dipole_fp64(tp, orc, alg):
    w, prob, keep = _regular_dipole(tp, 256, 2000, 50)
    w.tend = w.tend[keep]
    a = tp.AdaptiveBoris(0.1) if alg == "adaptive" else tp.AdaptiveMultistepBoris(4, 2, 0.1)
    sols, ref = _both(tp, orc, prob, a, tend=w.tend, savestepinterval=w.savestepinterval,
                      isoutside=w.isoutside, step_cap=2000)
    _check_same_layout(sols, ref)      # identical step decisions
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel(sols.u_all, ref.u) <= 1e-13


def test_adaptive_reference_kat_gpu(tp):
    # test_boris.jl:212-248 through the B200 path (gradient B = AffineField)
    tperiod = abs(tp.get_gyroperiod(0.01, q=tp.qe, m=tp.me))
    E = tp.UniformField((0.0, 1.0e5, 0.0))
    B = tp.AffineField((0.0, 0.0, 0.01), ((0, 0, 0), (0, 0, 0), (0.01, 0, 0)))
    prob = tp.TraceProblem([0.0, 0.0, 0.0, 1.0e7, 0.0, 0.0], (0.0, 200 * tperiod),
                           tp.prepare(E, B, species=tp.Electron))
    sol = tp.solve(prob, tp.AdaptiveBoris(0.1)).u[0]
    assert sol.t[-2] - sol.t[-3] < 0.8 * (sol.t[10] - sol.t[9])


def test_termination_boris_gpu(tp, orc):
    # test_boundary.jl:10-58 with the NaN region replaced by the shell predicate
    p = (1.0, 1.0, tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0)), tp.ZeroField())
    prob = tp.TraceProblem([0.9, 0.0, 0.0, 0.0, 1.0, 0.0], (0.0, 1.0), p)
    out = tp.TerminateNaN() | tp.TerminateShell(rmax=1.0)
    for alg, kw in ((tp.Boris(), dict(dt=0.2)), (tp.AdaptiveBoris(0.05), {})):
        sols, ref = _both(tp, orc, prob, alg, isoutside=out, **kw)
        _check_same_layout(sols, ref)
        sol = sols.u[0]
        assert sol.retcode == "Terminated" and np.linalg.norm(sol.u[-1][:3]) <= 1.0
        assert _rel(sols.u_all, ref.u) <= 1e-13


def test_queue_and_static_schedules_agree(tp):
    w = tp.workloads.config3(512, nt=1000, ssi=250)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B))
    kw = dict(dt=w.dt, tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    a = tp.solve(prob, tp.MultistepBoris(4, 2), tp.EnsembleB200(schedule="static"), **kw)
    b = tp.solve(prob, tp.MultistepBoris(4, 2), tp.EnsembleB200(schedule="queue"), **kw)
    assert np.array_equal(a.nsaved, b.nsaved) and np.array_equal(a.u_all, b.u_all)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_two_particles_per_thread_is_the_same_solve(tp, precision):
    # particles advanced two per thread in lock step take the same arithmetic
    # as one per thread: identical saves, step counts and return codes, with
    # either schedule and for a particle count that leaves a slot empty
    w = tp.workloads.config3(1001, nt=1500, ssi=250)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B))
    kw = dict(dt=w.dt, tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    for alg in (tp.MultistepBoris(4, 2), tp.Boris()):
        ref = tp.solve(prob, alg, tp.EnsembleB200(precision=precision, particles_per_thread=1, schedule="static"),
                       **kw)
        for sched in ("static", "queue"):
            s = tp.solve(prob, alg, tp.EnsembleB200(precision=precision, particles_per_thread=2, schedule=sched),
                         **kw)
            assert np.array_equal(s.nsaved, ref.nsaved) and np.array_equal(s.retcodes, ref.retcodes)
            assert np.array_equal(s.nsteps, ref.nsteps)
            assert np.array_equal(s.t_all, ref.t_all) and np.array_equal(s.u_all, ref.u_all)


# ------------------------------------------------------------------ gridded fields
def _small_grid_workload(tp, n=512, nx=32, nt=2000, ssi=500):
    dx = 1.0e5
    Ea, Ba, L = tp.workloads.turbulent_grid(nx, dx, 5.0e-9, nmodes=16)
    E = tp.FieldInterpolator(Ea, (0.0, 0.0, 0.0), (dx,) * 3, tp.WrapExtrap())
    B = tp.FieldInterpolator(Ba, (0.0, 0.0, 0.0), (dx,) * 3, tp.WrapExtrap())
    rng = tp.workloads.SplitMix64(99)
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(3 * n, 0.0, L).reshape(3, n)
    u0[3:] = rng.normal(3 * n, 2.0e5 / math.sqrt(2)).reshape(3, n)
    dt = tp.get_gyroperiod(5.0e-9) / 50
    return tp.TraceProblem(u0, (0.0, nt * dt), tp.prepare(E, B)), dt, ssi


def test_grid_boris_fp64_matches_oracle(tp, orc):
    prob, dt, ssi = _small_grid_workload(tp)
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=dt, savestepinterval=ssi)
    _check_same_layout(sols, ref)
    assert np.array_equal(sols.t_all, ref.t)
    assert _rel(sols.u_all, ref.u) <= 1e-13


@pytest.mark.parametrize("bc", ["fill", "clamp"])
def test_grid_boundaries_fp64(tp, orc, bc):
    # separate E / B tables (E uniform), non-periodic boundary rules
    dx = 1.0e5
    _, Ba, L = tp.workloads.turbulent_grid(16, dx, 5.0e-9, nmodes=8)
    b = tp.FillExtrap() if bc == "fill" else tp.ClampExtrap()
    B = tp.FieldInterpolator(Ba, (0.0, 0.0, 0.0), (dx,) * 3, b)
    rng = tp.workloads.SplitMix64(7)
    n = 256
    u0 = np.empty((6, n))
    u0[:3] = rng.uniform(3 * n, 0.2 * L, 0.8 * L).reshape(3, n)
    u0[3:] = rng.normal(3 * n, 1.0e5).reshape(3, n)
    dt = tp.get_gyroperiod(5.0e-9) / 50
    prob = tp.TraceProblem(u0, (0.0, 1000 * dt), tp.prepare(tp.UniformField((0.0, 1e-4, 0.0)), B))
    out = tp.TerminateNaN() if bc == "fill" else None
    sols, ref = _both(tp, orc, prob, tp.Boris(), dt=dt, savestepinterval=100, isoutside=out)
    _check_same_layout(sols, ref)
    assert _rel(sols.u_all, ref.u) <= 1e-13


def test_grid_fp32c_error_stated(tp, orc):
    # One gyroperiod (50 steps) in the turbulent field, before the chaotic
    # divergence of neighbouring orbits dominates: float32 + compensation
    # tracks the float64 oracle to ~1e-6 of the position.  (Over 1e4 steps any
    # two precisions diverge; bench.py states that divergence next to the one
    # between two float64 runs started 1 ulp apart.)
    prob, dt, ssi = _small_grid_workload(tp, nt=50, ssi=10)
    sols = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=dt, savestepinterval=ssi)
    plan = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(), dt=dt, savestepinterval=ssi)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
    assert np.array_equal(sols.nsaved, ref.nsaved)
    assert _pos_rel(sols.u_all, ref.u) <= 1e-5


# ------------------------------------------------------------------ FP32C in analytic fields
def test_fp32c_uniform(tp, orc):
    w = tp.workloads.config1(1000)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B))
    sols = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt,
                    savestepinterval=w.savestepinterval)
    plan = tp.plan_boris(prob, tp.Boris(), dt=w.dt, savestepinterval=w.savestepinterval)
    ref = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0)
    assert np.array_equal(sols.nsaved, ref.nsaved)
    # positions are O(1 m) displacements around O(1e6 m) gyro-orbits: compare on the orbit scale
    d = np.abs(sols.u_all[:, :3] - ref.u[:, :3]).max()
    assert d <= 1e-5 * np.abs(ref.u[:, :3]).max()


def _saves_by_particle(sols, nslots):
    """(n, nslots, 3) saved positions of particles that made every save, and that mask."""
    full = sols.nsaved == nslots
    off = np.concatenate([[0], np.cumsum(sols.nsaved.astype(np.int64))])
    rows = off[:-1][full][:, None] + np.arange(nslots)[None, :]
    return sols.u_all[rows, :3], full


def test_fp32c_dipole_multistep_error_bar(tp):
    """The FP32C bar on the dipole ensemble: MultistepBoris4(2), 1e4 steps, a
    fixed 4096-particle sample of the 1e6-proton workload (every 4th particle).
    The float64 runs started a float32 ulp away (components rounded to
    float32; all scaled by 1 + 2^-23) measure each orbit's own sensitivity:
      p90 of the final-position error over all orbits <= 1e-5;
      every regular orbit (both float32-ulp starts within 1e-6 / 1e-5 of the
      float64 orbit at every save) <= 1e-5."""
    w = tp.workloads.config3()
    idx = np.arange(0, 4 * 4096, 4)
    u0, dt, tend = w.u0[:, idx].copy(), w.dt[idx].copy(), w.tend[idx].copy()
    param = tp.prepare(w.E, w.B, species=tp.Proton)
    kw = dict(dt=dt, tend=tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    nslots = w.nt // w.savestepinterval + 1

    def run(u, prec):
        return tp.solve(tp.TraceProblem(u, w.tspan, param), tp.MultistepBoris4(2), tp.EnsembleB200(precision=prec),
                        **kw)

    x32, f32 = _saves_by_particle(run(u0, "fp32c"), nslots)
    s64 = run(u0, "fp64")
    x64, f64 = _saves_by_particle(s64, nslots)
    xr, fr = _saves_by_particle(run(u0.astype(np.float32).astype(np.float64), "fp64"), nslots)
    xs, fs = _saves_by_particle(run(u0 * (1.0 + 2.0 ** -23), "fp64"), nslots)
    both = f32 & f64 & fr & fs
    assert both.mean() > 0.95

    def sel(x, f):  # rows of the particles in `both`
        pos = np.cumsum(f) - 1
        return x[pos[both]]

    a64 = sel(x64, f64)

    def err(x, f):
        return np.linalg.norm(sel(x, f) - a64, axis=2) / np.linalg.norm(a64, axis=2)

    e32 = err(x32, f32)[:, -1]
    sr, ss = err(xr, fr).max(axis=1), err(xs, fs).max(axis=1)
    regular = (sr < 1e-6) & (ss < 1e-5)
    print(f"FP32C error: p50 {np.median(e32):.2e} p90 {np.quantile(e32, 0.9):.2e}; regular orbits "
          f"{regular.mean():.2f}, max {e32[regular].max():.2e}")
    assert np.quantile(e32, 0.9) <= 1e-5
    assert regular.mean() > 0.4
    assert e32[regular].max() <= 1e-5


# ------------------------------------------------------------------ guiding centre
def _gc_dipole(tp, orc):
    Ek = 5.0e7
    v0 = tp.sph2cart(tp.energy2velocity(Ek), math.pi / 4, 0.0)
    r0 = tp.sph2cart(2.5 * tp.Re, math.pi / 2, 0.0)
    E, B = tp.ZeroField(), tp.DipoleField(tp.BMoment_Earth)
    y0, p = tp.prepare_gc(np.concatenate([r0, v0]), E, B, species=tp.Proton)
    y0o, muo = orc.gc_prepare(E, B, np.concatenate([r0, v0]), tp.qi, tp.mi)
    assert _rel(y0, y0o[0]) <= 1e-14 and abs(p[2] - muo[0]) <= 1e-14 * muo[0]
    return tp.TraceGCProblem(y0, (0.0, 1.0), p)


def test_gc_full_conversion_gpu(tp, orc):
    # test_gc.jl:62-160 through the device (full_to_gc = tp_gc_prepare, gc_to_full = tp_gc_to_full)
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 1.0)), species=tp.Proton)
    R, vpar, mu = np.array([1.0, 0.0, 0.0]), 1.0e5, 1.0e-15
    xu = tp.gc_to_full(np.r_[R, vpar], param, mu, np.pi / 3)
    assert xu.shape == (6,)
    y, mu_new = tp.full_to_gc(xu, param)
    assert np.allclose(y[:3], R, rtol=1e-5) and np.isclose(y[3], vpar, rtol=1e-5) and np.isclose(mu_new, mu, rtol=1e-5)
    param2 = tp.prepare(tp.UniformField((0.0, 1.0e3, 0.0)), tp.UniformField((0.0, 0.0, 1.0)), species=tp.Proton)
    xu = tp.gc_to_full(np.zeros(4), param2, 0.0)
    assert np.allclose(xu[3:], [1000.0, 0.0, 0.0], atol=1e-5)
    y, mu_new = tp.full_to_gc(xu, param2)
    assert np.allclose(y, 0.0, atol=1e-5) and abs(mu_new) <= 1e-10
    v0 = tp.gc_to_full(np.zeros(4), param, 1.0e-15, 0.0)[3:]
    v90 = tp.gc_to_full(np.zeros(4), param, 1.0e-15, np.pi / 2)[3:]
    assert np.allclose(v0 / np.linalg.norm(v0), [1, 0, 0], atol=1e-5)
    assert np.allclose(v90 / np.linalg.norm(v90), [0, 1, 0], atol=1e-5)
    # parity with the oracle on guiding centres in the dipole, per-particle phase
    w = tp.workloads.config4(256)
    keep = slice(128, 256)  # the protons
    y = w.y0[:, keep]
    rng = np.random.default_rng(11)
    ph = rng.uniform(0.0, 2 * np.pi, y.shape[1])
    pd = tp.prepare(w.E, w.B, species=tp.Proton)
    xv = tp.gc_to_full(y, pd, w.mu[keep], ph)
    ref = orc.gc_to_full(w.E, w.B, y.T, w.mu[keep], tp.Proton.q, tp.Proton.m, ph)
    assert xv.shape == (6, 128)
    assert _rel(xv.T, ref) <= 1e-13
    yb, mub = tp.full_to_gc(xv, pd)
    yr, mur = orc.gc_prepare(w.E, w.B, ref, tp.Proton.q, tp.Proton.m)
    assert _rel(yb.T, yr) <= 1e-13 and np.max(np.abs(mub - mur) / mur) <= 1e-13


def test_gc_reference_counts_gpu(tp, orc):
    # test_gc.jl:190-251 through the B200 path
    prob = _gc_dipole(tp, orc)
    s = tp.solve(prob, dt=1.0e-4, alg="rk4").u[0]
    assert len(s.t) == 10001 and s.retcode == "MaxIters"
    assert len(tp.solve(prob, dt=1.0e-4, alg="rk4", save_everystep=False).u[0].t) == 2
    assert len(tp.solve(prob, dt=1.0e-4, alg="rk4", isoutside=tp.TerminateTime(0.5)).u[0].t) == 5001
    s = tp.solve(prob, dt=1.0e-4, alg="rk45").u[0]
    assert len(s.t) == 61 and s.retcode == "Success"
    s = tp.solve(prob, alg="rk45").u[0]
    assert len(s.t) == 58 and s.retcode == "Success"


@pytest.mark.parametrize("alg", ["rk4", "rk45"])
def test_gc_fp64_matches_oracle(tp, orc, alg):
    prob = _gc_dipole(tp, orc)
    kw = dict(dt=1.0e-4, alg=alg)
    sols = tp.solve(prob, **kw)
    plan = tp.plan_gc(prob, **kw)
    ref = orc.gc_run(plan.desc, plan.E, plan.B, plan.y0)
    _check_same_layout(sols, ref)
    if alg == "rk4":
        assert np.array_equal(sols.t_all, ref.t)
        assert _rel(sols.u_all, ref.u) <= 1e-13
    else:
        # the step controller's pow() (CUDA vs glibc) may differ in the last bit
        assert _rel(sols.t_all, ref.t) <= 1e-10
        assert _rel(sols.u_all, ref.u) <= 1e-10


@pytest.mark.parametrize("alg", ["rk4", "rk45"])
def test_gc_save_fields_and_work(tp, orc, alg):
    # test_gc.jl:268-304 shape, plus parity of every saved column
    prob = _gc_dipole(tp, orc)
    kw = dict(dt=1.0e-4, alg=alg, save_fields=True, save_work=True, maxiters=2000)
    sols = tp.solve(prob, **kw)
    plan = tp.plan_gc(prob, **kw)
    ref = orc.gc_run(plan.desc, plan.E, plan.B, plan.y0)
    _check_same_layout(sols, ref)
    assert sols.u_all.shape[1] == 14
    assert np.linalg.norm(sols.u_all[0, 7:10]) > 0.0 and np.all(sols.u_all[:, 4:7] == 0.0)
    assert np.all(sols.u_all[:, 10:14] == 0.0)   # E = 0 and static B
    assert _rel(sols.u_all, ref.u) <= (1e-13 if alg == "rk4" else 1e-10)


def test_gc_config4_subset(tp, orc):
    w = tp.workloads.config4(512)
    prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
    dt = w.tau_b / 200
    kw = dict(dt=dt, tend=5 * w.tau_b, alg="rk4", savestepinterval=100)
    sols = tp.solve(prob, **kw)
    plan = tp.plan_gc(prob, **kw)
    ref = orc.gc_run(plan.desc, plan.E, plan.B, plan.y0, plan.q_i, plan.q2m_i, plan.mu_i,
                     dt_i=plan.dt_i, tend_i=plan.tend_i)
    _check_same_layout(sols, ref)
    assert _rel(sols.u_all, ref.u) <= 1e-12
    s32 = tp.solve(prob, tp.EnsembleB200(precision="fp32"), **kw)
    assert np.array_equal(s32.nsaved, ref.nsaved)
    err = np.linalg.norm(s32.final_states()[:, :3] - ref.final_states()[:, :3], axis=1) / \
        np.linalg.norm(ref.final_states()[:, :3], axis=1)
    assert np.median(err) <= 1e-4


# ---------------------------------------------------------------- tuning and graphs
def test_autotune_chooses_a_valid_shape_and_keeps_results(tp):
    w = tp.workloads.config2(n=20000, nt=300, ssi=100)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    base = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt, savestepinterval=100)
    plan = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt, savestepinterval=100)
    ctx = tp.Context.get(0)
    r = ctx.autotune(plan.desc, plan.E, plan.B, plan.u0, max_steps=100)
    assert r["block"] in (64, 96, 128, 192, 256, 384) and r["schedule"] in ("static", "queue")
    assert r["candidates"] >= 10 and 0 < r["ms"] <= 1.25 * r["ms_default"]
    tuned = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt, savestepinterval=100)
    # per-particle arithmetic does not depend on the launch shape
    assert np.array_equal(tuned.u_all, base.u_all) and np.array_equal(tuned.t_all, base.t_all)
    auto = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c", autotune=True), dt=w.dt,
                    savestepinterval=100)
    assert np.array_equal(auto.u_all, base.u_all)
    assert r["particles_per_thread"] == 1  # grids: one particle per thread only


def test_autotune_times_particles_per_thread_in_analytic_fields(tp):
    w = tp.workloads.config3(n=60000, nt=300, ssi=100)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    kw = dict(dt=w.dt, tend=w.tend, savestepinterval=100)
    ctx = tp.Context.get(0)
    for prec in ("fp32c", "fp64"):
        plan = tp.plan_boris(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision=prec), **kw)
        base = tp.solve(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision=prec, particles_per_thread=1),
                        **kw)
        r = ctx.autotune(plan.desc, plan.E, plan.B, plan.u0, max_steps=100)
        assert r["particles_per_thread"] in (1, 2)
        assert r["candidates"] >= 18  # (block sizes x schedules) for one and for two particles per thread
        tuned = tp.solve(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision=prec), **kw)
        assert np.array_equal(tuned.u_all, base.u_all)


@pytest.mark.parametrize("term", [False, True])
def test_graph_replay_equals_direct_run(tp, term):
    import torch
    w = tp.workloads.config3(n=4096, nt=500, ssi=100)
    isout = w.isoutside if term else None
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp32c"), dt=w.dt,
                         savestepinterval=100, isoutside=isout, tend=w.tend)
    ctx = tp.Context.get(0)
    n = plan.u0.shape[0]
    nslots = ctx.slots(plan.desc, n, plan.dt_i, plan.tend_i)
    dev = torch.device("cuda", 0)
    f = lambda a: None if a is None else torch.from_numpy(a).to(dev)  # noqa: E731
    u0, dt_i, tend_i = f(plan.u0), f(plan.dt_i), f(plan.tend_i)

    def bufs():
        return (torch.full((nslots, n), np.nan, dtype=torch.float64, device=dev),
                torch.full((nslots, 6, n), np.nan, dtype=torch.float64, device=dev),
                torch.zeros(n, dtype=torch.int32, device=dev), torch.zeros(n, dtype=torch.int8, device=dev),
                torch.zeros(n, dtype=torch.int64, device=dev), torch.zeros(1, dtype=torch.int32, device=dev))

    p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    a = bufs()
    ctx.boris_run_device(plan.desc, plan.E, plan.B, p(u0), p(dt_i), p(tend_i), n, nslots, *[p(x) for x in a],
                         torch.cuda.current_stream().cuda_stream)
    b = bufs()
    g = ctx.boris_graph(plan.desc, plan.E, plan.B, p(u0), p(dt_i), p(tend_i), n, nslots, *[p(x) for x in b])
    for _ in range(2):  # replays rewrite the same buffers
        g.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(torch.nan_to_num(x, nan=7.0), torch.nan_to_num(y, nan=7.0))
    g.close()
