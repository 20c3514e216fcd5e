"""tp_pack_results_device_noalloc: packing that allocates no device memory.

Some callers cannot let a library call cudaMalloc: their own memory pool owns
every device buffer, or allocation is forbidden on their latency path.  For
them the library packs device-resident results through a static scratch array
instead.  This test runs a solve through the device entry point into caller
buffers, packs it with the no-allocation entry point, and checks the result
against the allocating host entry point (tp_boris_run) -- bit for bit, since
both run the same kernels on the same inputs -- on two calls in a row.  The
file sorts last so that a run stopping at the first failure has already run
every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(tp, kind, n=None):
    if kind == "fixed":
        w = tp.workloads.config1(n or 300)
        prob = tp.TraceProblem(w.u0, (0.0, 2000 * w.dt), tp.prepare(w.E, w.B))
        return tp.plan_boris(prob, tp.Boris(), dt=w.dt, savestepinterval=100)
    # adaptive steps in the dipole: the save counts differ from particle to
    # particle, so every trajectory's packed offset depends on all before it
    nt, ssi = (500, 40) if n is None else (120, 10)
    w = tp.workloads.config3(n or 200, nt=nt, ssi=ssi)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B))
    return tp.plan_boris(prob, tp.AdaptiveBoris(0.1), tend=w.tend, savestepinterval=ssi, isoutside=w.isoutside,
                         step_cap=nt)


def _pack_without_alloc(tp, torch, ctx, plan):
    n = plan.u0.shape[0]
    nslots = ctx.slots(plan.desc, n, plan.dt_i, plan.tend_i)
    W = 6 + 6 * bool(plan.desc.save_fields) + 4 * bool(plan.desc.save_work)
    dev = torch.device("cuda", 0)
    u0 = torch.from_numpy(plan.u0).to(dev)
    dti = None if plan.dt_i is None else torch.from_numpy(plan.dt_i).to(dev)
    tend = None if plan.tend_i is None else torch.from_numpy(plan.tend_i).to(dev)
    t_sm = torch.empty((nslots, n), dtype=torch.float64, device=dev)
    u_sm = torch.empty((nslots, W, n), dtype=torch.float64, device=dev)
    nsaved = torch.empty(n, dtype=torch.int32, device=dev)
    retc = torch.empty(n, dtype=torch.int8, device=dev)
    nsteps = torch.empty(n, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    stream = torch.cuda.current_stream().cuda_stream
    ctx.boris_run_device(plan.desc, plan.E, plan.B, p(u0), p(dti), p(tend), n, nslots, p(t_sm), p(u_sm),
                         p(nsaved), p(retc), p(nsteps), p(status), stream)
    # packed outputs sized for the worst case; NaN marks what the call did not write
    t_pk = torch.full((n * nslots,), float("nan"), dtype=torch.float64, device=dev)
    u_pk = torch.full((n * nslots, W), float("nan"), dtype=torch.float64, device=dev)
    total = torch.full((1,), -1, dtype=torch.int64, device=dev)
    code = ctx.lib.tp_pack_results_device_noalloc(ctx.handle, p(t_sm), p(u_sm), p(nsaved), n, nslots, W,
                                                  p(t_pk), p(u_pk), p(total), stream)
    assert code == tp._abi.TP_OK, ctx.lib.tp_last_error(ctx.handle)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    tot = int(total.item())
    ns = nsaved.cpu().numpy()
    # the reported total is the sum of the clamped save counts
    assert tot == int(np.minimum(np.maximum(ns.astype(np.int64), 0), nslots).sum())
    return ns, t_pk[:tot].cpu().numpy(), u_pk[:tot].cpu().numpy(), t_pk[tot:].cpu().numpy()


def _check_against_allocating_path(tp, torch, ctx, plan):
    ref = ctx.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i, pipelined=False)
    nsaved, t, u, rest = _pack_without_alloc(tp, torch, ctx, plan)
    assert np.array_equal(nsaved, ref.nsaved)
    assert t.shape == ref.t.shape and u.shape == ref.u.shape
    assert np.array_equal(t, ref.t)
    assert np.array_equal(u, ref.u, equal_nan=True)
    assert np.all(np.isnan(rest))  # nothing written past the packed total
    return nsaved


def test_noalloc_pack_matches_allocating_entry_point(tp):
    torch = pytest.importorskip("torch")
    ctx = tp.Context.get(0)
    for kind in ("fixed", "adaptive"):  # two calls in a row share the static scratch
        _check_against_allocating_path(tp, torch, ctx, _problem(tp, kind))


@pytest.mark.parametrize("n", [5000, 1048576])
def test_noalloc_pack_across_scan_blocks(tp, n):
    """Several 1024-trajectory scan blocks, uneven save counts, and the largest n
    the static scratch takes: every block's offset comes from the scan of the
    block totals, so a wrong block prefix shows up as a mismatch."""
    torch = pytest.importorskip("torch")
    assert n <= tp._abi.TP_NOALLOC_MAX_TRAJECTORIES
    ctx = tp.Context.get(0)
    nsaved = _check_against_allocating_path(tp, torch, ctx, _problem(tp, "adaptive", n))
    assert len(np.unique(nsaved)) > 1  # uneven: offsets are not a multiple of one count


def test_noalloc_pack_rejects_more_than_the_static_limit(tp):
    ctx = tp.Context.get(0)
    n = tp._abi.TP_NOALLOC_MAX_TRAJECTORIES + 1
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    code = ctx.lib.tp_pack_results_device_noalloc(ctx.handle, dummy, dummy, dummy, n, 1, 6, dummy, dummy, dummy,
                                                  None)
    assert code == tp._abi.TP_E_ARG
    assert b"static scratch limit" in ctx.lib.tp_last_error(ctx.handle)
