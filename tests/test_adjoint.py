"""Discrete adjoint of the Boris map.

The oracle's forward-mode tangent (orc_boris_jvp) stands in for ForwardDiff
through the reference solver.  It is pinned by (CPU tests):
  * its primal equals the final save of the oracle's Boris solve, bit for bit;
  * central finite differences with relative step 1e-4 in smooth (analytic)
    fields;
  * central finite differences in the trilinear config-2 field.  That field
    is only continuous, so the map's derivative jumps wherever a step's
    position crosses a cell face.  A relative step of 1e-4 (1 km on 1e7 m
    coordinates, 1 % of a cell) straddles such crossings in most
    trajectories.  The check therefore uses small steps and particles whose
    difference quotients agree at two step sizes.
The GPU adjoint (tp_adjoint_*) is then compared with the tangent at 1e-4
relative.  That is a vector-Jacobian product against Jacobian-vector
products along the same directions, with the same cotangent.
"""
from __future__ import annotations

import numpy as np
import pytest


def _grid_case(tp, n=16, nt=256):
    w = tp.workloads.config5(n=n, nt=nt)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    return w, prob


def _desc(tp, prob, dt):
    return tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(), dt=dt, savestepinterval=1,
                         save_start=False, save_everystep=False)


def _smooth_case(tp, n=16, nt=256):
    """Protons in an Earth dipole plus a uniform-offset affine E (smooth fields)."""
    rng = np.random.default_rng(5)
    L = rng.uniform(3.0, 5.0, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    r = np.stack([L * tp.Re * np.cos(phi), L * tp.Re * np.sin(phi), rng.uniform(-0.2, 0.2, n) * tp.Re])
    v = rng.normal(size=(3, n)) * 2.0e6
    u0 = np.concatenate([r, v])
    B = tp.DipoleField((0.0, 0.0, -8.0e22))
    E = tp.AffineField((1.0e-3, -2.0e-4, 5.0e-4), ((0.0, 1.0e-10, 0.0), (-1.0e-10, 0.0, 0.0), (0.0, 0.0, 2.0e-11)))
    Bmag = 3.1e-5 / np.min(L) ** 3
    dt = tp.get_gyroperiod(Bmag) / 50
    prob = tp.TraceProblem(u0, (0.0, nt * dt), tp.prepare(E, B, species=tp.Proton))
    return prob, E, B, dt


# ---------------------------------------------------------------- CPU: oracle
def test_oracle_tangent_primal_is_the_boris_solve(tp, orc):
    w, prob = _grid_case(tp, n=8, nt=64)
    p = _desc(tp, prob, w.dt)
    uN, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0)
    ref = orc.boris_run(p.desc, p.E, p.B, p.u0)
    off = np.zeros(ref.nsaved.size + 1, dtype=np.int64)
    np.cumsum(ref.nsaved, out=off[1:])
    assert np.array_equal(ref.u[off[1:] - 1], uN)


def test_oracle_tangent_vs_central_differences_smooth(tp, orc):
    prob, E, B, dt = _smooth_case(tp, n=8, nt=128)
    p = _desc(tp, prob, dt)
    rng = np.random.default_rng(1)
    d = rng.normal(size=p.u0.shape) * np.abs(p.u0)
    uN, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, du0=d)
    rel = 1.0e-4
    up, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0 + rel * d)
    um, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0 - rel * d)
    fd = (up - um) / (2 * rel)
    err = np.linalg.norm(fd - dN, axis=1) / np.linalg.norm(dN, axis=1)
    assert err.max() <= 1.0e-4, err  # O(h^2) truncation of the central difference
    # parameters: dipole moment and the affine field's constant term
    dp = np.array([1.0e-4, -3.0e-4, 2.0e-4, 1.0e21, -2.0e21, 3.0e21])
    _, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, dparam=dp)
    h = 1.0e-4

    def shifted(s):
        Es = tp.AffineField(tuple(np.add(E.value, s * dp[:3])), E.jac)
        Bs = tp.DipoleField(tuple(np.add(B.moment, s * dp[3:])))
        return orc.boris_jvp(p.desc, Es, Bs, p.u0)[0]

    fd = (shifted(h) - shifted(-h)) / (2 * h)
    err = np.linalg.norm(fd - dN, axis=1) / np.linalg.norm(dN, axis=1)
    assert err.max() <= 1.0e-4, err


def test_oracle_tangent_vs_central_differences_grid(tp, orc):
    w, prob = _grid_case(tp, n=16, nt=256)
    p = _desc(tp, prob, w.dt)
    rng = np.random.default_rng(2)
    d = rng.normal(size=p.u0.shape) * np.abs(p.u0)
    _, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, du0=d)

    def fd(rel):
        up, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0 + rel * d)
        um, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0 - rel * d)
        return (up - um) / (2 * rel)

    f1, f2 = fd(1.0e-8), fd(2.0e-8)
    scale = np.linalg.norm(dN, axis=1)
    clean = np.linalg.norm(f1 - f2, axis=1) <= 1.0e-6 * scale  # no face crossing inside the step
    assert clean.sum() >= 12
    err = np.linalg.norm(f1 - dN, axis=1) / scale
    assert np.all(err[clean] <= 1.0e-5), err
    # the relative step 1e-4 straddles face crossings: report, do not assert
    e4 = np.linalg.norm(fd(1.0e-4) - dN, axis=1) / scale
    print(f"central differences at relative step 1e-4: median rel. err {np.median(e4):.2e} (cell-face kinks)")


# ---------------------------------------------------------------- GPU
def _per_particle_vjp(orc, p, c):
    """J_i^T c_i of every particle from 6 forward tangents (particles are independent)."""
    n = p.u0.shape[0]
    out = np.empty((n, 6))
    for k in range(6):
        e = np.zeros((n, 6))
        e[:, k] = 1.0
        _, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, du0=e)
        out[:, k] = np.sum(c * dN, axis=1)
    return out


def _rel_rows(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.mark.gpu
def test_adjoint_forward_is_the_fp32c_solve(tp):
    w, prob = _grid_case(tp, n=256, nt=200)
    uf, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=64)
    sol = tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision="fp32c"), dt=w.dt, savestepinterval=10**6,
                   save_start=False)
    assert np.array_equal(sol.final_states(), uf)
    bytes_, nsteps = tape.info()
    assert nsteps == 200 and bytes_ > 0


@pytest.mark.gpu
def test_adjoint_grid_vs_oracle_tangent(tp, orc):
    w, prob = _grid_case(tp, n=16, nt=256)
    p = _desc(tp, prob, w.dt)
    uN, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0)
    x_target = uN[:, :3] + w.extra["target_offset"]
    _, c = tp.workloads.loss_and_grad(uN, x_target)  # same cotangent for both sides

    uf, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=64)
    dev = np.linalg.norm(uf[:, :3] - uN[:, :3], axis=1) / np.linalg.norm(uN[:, :3], axis=1)
    g = tape.backward(c)

    ref = _per_particle_vjp(orc, p, c)
    err = _rel_rows(g.u0, ref)
    print("FP32C-vs-FP64 final position deviation:", np.array2string(dev, precision=2))
    print("dL/du0 relative error per particle:   ", np.array2string(err, precision=2))
    assert np.all(err <= 1.0e-4), err

    # node values along random directions
    rng = np.random.default_rng(3)
    for _ in range(2):
        dE = rng.normal(size=w.E.data.shape) * 2.0e-3
        dB = rng.normal(size=w.B.data.shape) * 5.0e-9
        _, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, dE_nodes=dE, dB_nodes=dB)
        s_ref = float(np.sum(c * dN))
        s_gpu = float(np.sum(g.E.astype(np.float64) * dE) + np.sum(g.B.astype(np.float64) * dB))
        assert abs(s_gpu - s_ref) <= 1.0e-4 * abs(s_ref), (s_gpu, s_ref)

    # B0: B_z = B0 + dB_z at every node and E_y = u_x B_z
    ux = 4.0e5
    _, dN = orc.boris_jvp(p.desc, p.E, p.B, p.u0, dparam=[0.0, ux, 0.0, 0.0, 0.0, 1.0])
    dLdB0_ref = float(np.sum(c * dN))
    dLdB0 = ux * g.param[1] + g.param[5]
    assert abs(dLdB0 - dLdB0_ref) <= 1.0e-4 * abs(dLdB0_ref)
    # the offset gradients are the node-gradient sums
    assert np.allclose(g.param[:3], g.E.reshape(3, -1, order="F").sum(axis=1, dtype=np.float64), rtol=1e-5,
                       atol=1e-12 * np.abs(g.param[:3]).max())


@pytest.mark.gpu
def test_adjoint_smooth_fields_vs_central_differences(tp, orc):
    prob, E, B, dt = _smooth_case(tp, n=16, nt=256)
    p = _desc(tp, prob, dt)
    uN, _ = orc.boris_jvp(p.desc, p.E, p.B, p.u0)
    rng = np.random.default_rng(4)
    c = rng.normal(size=uN.shape) * np.array([1e-7, 1e-7, 1e-7, 1e-6, 1e-6, 1e-6])
    uf, tape = tp.adjoint_solve(prob, dt=dt)
    g = tape.backward(c)
    # u0 against central differences of the oracle (relative step 1e-4)
    n = uN.shape[0]
    ref = np.empty((n, 6))
    rmag = np.linalg.norm(p.u0[:, :3], axis=1)
    vmag = np.linalg.norm(p.u0[:, 3:], axis=1)
    for k in range(6):
        h = 1.0e-4 * (rmag if k < 3 else vmag)  # relative step 1e-4 of the vector
        up, um = p.u0.copy(), p.u0.copy()
        up[:, k] += h
        um[:, k] -= h
        fp, _ = orc.boris_jvp(p.desc, p.E, p.B, up)
        fm, _ = orc.boris_jvp(p.desc, p.E, p.B, um)
        ref[:, k] = np.sum(c * (fp - fm), axis=1) / (2 * h)
    assert np.all(_rel_rows(g.u0, ref) <= 1.0e-4), _rel_rows(g.u0, ref)
    # dipole moment and the affine constant term against central differences
    for k in range(6):
        dp = np.zeros(6)
        h = 1.0e-4 * (np.linalg.norm(E.value) if k < 3 else np.linalg.norm(B.moment))
        dp[k] = h
        Ep = tp.AffineField(tuple(np.add(E.value, dp[:3])), E.jac)
        Bp = tp.DipoleField(tuple(np.add(B.moment, dp[3:])))
        Em = tp.AffineField(tuple(np.subtract(E.value, dp[:3])), E.jac)
        Bm = tp.DipoleField(tuple(np.subtract(B.moment, dp[3:])))
        fp, _ = orc.boris_jvp(p.desc, Ep, Bp, p.u0)
        fm, _ = orc.boris_jvp(p.desc, Em, Bm, p.u0)
        ref_k = float(np.sum(c * (fp - fm))) / (2 * h)
        assert abs(g.param[k] - ref_k) <= 1.0e-4 * abs(ref_k), (k, g.param[k], ref_k)


@pytest.mark.gpu
def test_adjoint_independent_of_checkpoint_interval(tp):
    """K <= 8 runs the one-kernel backward (records in shared memory), larger
    K the two kernels per segment; 200 particles leave a partial warp and a
    partial block."""
    w, prob = _grid_case(tp, n=200, nt=100)
    rng = np.random.default_rng(6)
    c = rng.normal(size=(200, 6)) * np.array([1e-7] * 3 + [1e-6] * 3)
    res = []
    for K in (1, 3, 4, 7, 8, 9, 64, 100, 1000):
        uf, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=K)
        res.append((uf, tape.backward(c)))
    for uf, g in res[1:]:
        assert np.array_equal(uf, res[0][0])
        assert np.array_equal(g.u0, res[0][1].u0)  # recomputation is exact
        assert np.allclose(g.B, res[0][1].B, rtol=1e-5, atol=1e-6 * np.abs(res[0][1].B).max())


@pytest.mark.gpu
def test_adjoint_automatic_segments(tp):
    """checkpoint_every = 0: 2-step segments (one-kernel backward) on the
    interleaved E/B grid, 64 for analytic fields; explicit K is kept."""
    w, prob = _grid_case(tp, n=64, nt=100)
    _, tape = tp.adjoint_solve(prob, dt=w.dt)
    assert tape.segments() == (2, 50)
    _, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=7)
    assert tape.segments() == (7, 15)
    sprob, _, _, dt = _smooth_case(tp, n=16, nt=200)
    _, tape = tp.adjoint_solve(sprob, dt=dt)
    assert tape.segments() == (64, 4)


@pytest.mark.gpu
def test_adjoint_warp_aggregation(tp):
    """Particles sharing a cell: the aggregated scatter equals the per-particle sum."""
    w, prob = _grid_case(tp, n=1, nt=50)
    c1 = np.array([[1e-7, -2e-7, 3e-7, 1e-6, 0.0, -1e-6]])
    _, tape = tp.adjoint_solve(prob, dt=w.dt)
    g1 = tape.backward(c1)
    for copies in (32, 4, 96):  # a full warp, a group of 4, three full warps
        u0 = np.repeat(w.u0, copies, axis=1)
        probk = tp.TraceProblem(u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
        _, tk = tp.adjoint_solve(probk, dt=w.dt)
        gk = tk.backward(np.repeat(c1, copies, axis=0))
        assert np.array_equal(gk.u0, np.repeat(g1.u0, copies, axis=0))
        scale = np.abs(g1.B).max() * copies
        assert np.allclose(gk.B, copies * g1.B.astype(np.float64), rtol=1e-5, atol=1e-6 * scale)
        assert np.allclose(gk.E, copies * g1.E.astype(np.float64), rtol=1e-5, atol=1e-6 * np.abs(g1.E).max() * copies)


@pytest.mark.gpu
def test_adjoint_argument_errors(tp):
    w, prob = _grid_case(tp, n=4, nt=10)
    with pytest.raises(NotImplementedError):
        tp.plan_adjoint(prob, tp.EnsembleB200(precision="fp64"), dt=w.dt)
    p = tp.plan_adjoint(prob, dt=w.dt)
    ctx = tp.Context.get(0)
    p.desc.run.alg = tp._abi.TP_ALG_MULTISTEP
    p.desc.run.order, p.desc.run.nsub = 4, 2
    with pytest.raises(NotImplementedError):
        ctx.adjoint_forward(p.desc, p.E, p.B, p.u0)
    p = tp.plan_adjoint(prob, dt=w.dt)
    p.desc.checkpoint_every = -1
    with pytest.raises(tp.ArgumentError):
        ctx.adjoint_forward(p.desc, p.E, p.B, p.u0)


@pytest.mark.gpu
def test_torch_autograd_function(tp):
    import torch

    from testparticle_b200.autograd import GridTensor, boris_final_state
    w, prob = _grid_case(tp, n=32, nt=64)
    dev = torch.device("cuda", 0)
    u0 = torch.tensor(w.u0.T.copy(), device=dev, requires_grad=True)
    Bt = torch.tensor(np.asarray(w.B.data), device=dev, requires_grad=True)
    Et = torch.tensor(np.asarray(w.E.data), device=dev, requires_grad=True)
    B0 = torch.tensor(5.0e-9, dtype=torch.float32, device=dev, requires_grad=True)
    zhat = torch.tensor([0.0, 0.0, 1.0], device=dev).view(3, 1, 1, 1)
    yhat = torch.tensor([0.0, 1.0, 0.0], device=dev).view(3, 1, 1, 1)
    ux = 4.0e5
    # B0 enters B_z at every node and E_y = u_x B_z
    Bf = GridTensor(Bt + (B0 - 5.0e-9) * zhat, w.B.origin, w.B.spacing)
    Ef = GridTensor(Et + ux * (B0 - 5.0e-9) * yhat, w.E.origin, w.E.spacing)
    q2m = tp.Proton.q / tp.Proton.m
    out = boris_final_state(u0, Ef, Bf, q2m=q2m, m=tp.Proton.m, dt=w.dt, tspan=w.tspan)
    x_target = out.detach()[:, :3] + torch.tensor(w.extra["target_offset"], device=dev)
    loss = ((out[:, :3] - x_target) ** 2).sum(dim=1).mean()
    loss.backward()
    # the same through the ctypes path
    uf, tape = tp.adjoint_solve(prob, dt=w.dt)
    assert np.array_equal(uf, out.detach().cpu().numpy())
    _, c = tp.workloads.loss_and_grad(uf, x_target.cpu().numpy())
    g = tape.backward(c)
    assert np.allclose(u0.grad.cpu().numpy(), g.u0, rtol=1e-12, atol=0)
    assert np.allclose(Bt.grad.cpu().numpy(), g.B, rtol=1e-5, atol=1e-6 * np.abs(g.B).max())
    dB0 = ux * g.param[1] + g.param[5]
    assert abs(B0.grad.item() - dB0) <= 1e-3 * abs(dB0)


@pytest.mark.gpu
def test_adjoint_chaotic_range(tp):
    """4096 steps in the turbulent field: cotangents grow by 1e18 to 1e27, beyond
    float32; the scaled frames keep every gradient finite and the result does
    not depend on the checkpoint interval."""
    w, prob = _grid_case(tp, n=64, nt=4096)
    rng = np.random.default_rng(8)
    c = rng.normal(size=(64, 6)) * np.array([1e-7] * 3 + [1e-6] * 3)
    out = []
    for K in (4, 64, 512):
        _, tape = tp.adjoint_solve(prob, dt=w.dt, checkpoint_every=K)
        out.append(tape.backward(c))
    g = out[0]
    for a in (g.u0, g.E, g.B, g.param):
        assert np.all(np.isfinite(a))
    assert np.abs(g.u0[:, :3]).max() > 1e10  # the growth is real
    for o in out[1:]:
        assert np.array_equal(g.u0, o.u0)
        assert np.allclose(g.B, o.B, rtol=1e-4, atol=1e-6 * np.abs(g.B).max())
