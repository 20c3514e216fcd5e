"""tp_boris_run_host: the host-to-host solve with the copy-out overlapped.

One kernel runs the ensemble and counts finished particles per chunk of
consecutive indices; the host copies and packs each finished chunk while the
kernel still runs.  The results must equal tp_boris_run + tp_result_copy bit
for bit: the same kernel runs on the same inputs, and only the packing
(host threads instead of a device pass) differs.  The cases use several
chunks, uneven save counts (termination, per-particle spans), the cell
ordering of gridded solves (chunks then finish out of order), saved fields
and work rates (chunks final only at the end), the static schedule, and two
calls in a row.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    for name in ("nsaved", "retcode", "nsteps"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert a.t.shape == b.t.shape and a.u.shape == b.u.shape
    assert np.array_equal(a.t, b.t)
    assert np.array_equal(a.u, b.u, equal_nan=True)


def _both(ctx, plan):
    args = (plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    return ctx.boris_run(*args, pipelined=True), ctx.boris_run(*args, pipelined=False)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_pipelined_dipole_ensemble(tp, precision):
    """Twelve chunks of the dipole ensemble: per-particle dt and span, and the
    1 / 15 R_E termination, so save counts and packed offsets differ."""
    n = 3 * 131072 + 777
    w = tp.workloads.config3(n, nt=300, ssi=40)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision=precision), dt=w.dt,
                         tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    ctx = tp.Context.get(0)
    a, b = _both(ctx, plan)
    _same(a, b)
    assert len(np.unique(a.nsaved)) > 1
    # a second call reuses the staging buffers and pool memory that still holds
    # the first call's chunk counts
    again, _ = _both(ctx, plan)
    _same(again, b)


def test_pipelined_gridded_with_fields_and_work(tp):
    """A Cartesian grid (particles processed in cell order, so chunks finish
    out of index order), with the saved fields and work rates (16 columns:
    a post-pass completes them, so chunks are copied after the launch)."""
    n = 2 * 131072 + 4321
    w = tp.workloads.config2(n, nx=32, nt=120, ssi=30)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt,
                         savestepinterval=w.savestepinterval, save_fields=True, save_work=True)
    ctx = tp.Context.get(0)
    a, b = _both(ctx, plan)
    assert a.u.shape[1] == 16
    _same(a, b)


def test_pipelined_gridded_cell_order(tp):
    """Cell-ordered processing without a post-pass: the device-packing branch."""
    n = 150_000
    w = tp.workloads.config2(n, nx=32, nt=100, ssi=20)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(precision="fp64"), dt=w.dt,
                         savestepinterval=w.savestepinterval)
    ctx = tp.Context.get(0)
    a, b = _both(ctx, plan)
    _same(a, b)
    again, _ = _both(ctx, plan)
    _same(again, b)


def test_pipelined_static_schedule(tp):
    n = 100_000
    w = tp.workloads.config3(n, nt=200, ssi=25)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c", schedule="static"), dt=w.dt,
                         tend=w.tend, savestepinterval=w.savestepinterval, isoutside=w.isoutside)
    ctx = tp.Context.get(0)
    a, b = _both(ctx, plan)
    _same(a, b)


def test_pipelined_adaptive_with_step_cap(tp):
    n = 2 * 131072 + 99
    w = tp.workloads.config3(n, nt=120, ssi=10)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    plan = tp.plan_boris(prob, tp.AdaptiveBoris(0.1), tend=w.tend, savestepinterval=10, isoutside=w.isoutside,
                         step_cap=120)
    ctx = tp.Context.get(0)
    a, b = _both(ctx, plan)
    _same(a, b)
    assert len(np.unique(a.nsaved)) > 1


def test_pipelined_rejects_unknown_save_counts_and_short_buffers(tp):
    ctx = tp.Context.get(0)
    w = tp.workloads.config3(64, nt=100, ssi=10)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    # adaptive without a step cap: the save count is unknown in advance
    plan = tp.plan_boris(prob, tp.AdaptiveBoris(0.1), tend=w.tend, savestepinterval=10, isoutside=w.isoutside)
    with pytest.raises(NotImplementedError):
        ctx.boris_run_host(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i, 64 * 100)
    # the public path falls back to tp_boris_run for it
    r = ctx.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i)
    assert r.t.size == int(r.nsaved.sum())
    # fixed steps into buffers that cannot hold the saves
    plan = tp.plan_boris(prob, tp.Boris(), dt=w.dt, tend=w.tend, savestepinterval=10)
    with pytest.raises(tp.ArgumentError):
        ctx.boris_run_host(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i, 5)
    code = ctx.lib.tp_boris_run_host(ctx.handle, C.byref(plan.desc), ctx.field(plan.E), ctx.field(plan.B),
                                     None, None, None, -1, 0, None, None, None, None, None,
                                     C.byref(C.c_int64()), None)
    assert code == tp._abi.TP_E_ARG
