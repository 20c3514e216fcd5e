"""GPU parity of the virtual detectors (tp_detect_*) against the CPU oracle
(ext/TestParticleMeshesExt.jl:98-491 restated), plus the reference's
known-answer cases through the device path.

Bars: crossing counts and the order of the crossing rows are exact; crossing
states and first crossings use +, -, *, /, sqrt and one fma on both sides and
match to 1e-13; flux totals are summed in a different order (a fixed-order
tree on the device, trajectory by trajectory in the reference) and match to
1e-12.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _line_sol(tp, x0, y0, vx, vy, z0=0.0, vz=0.0, n=21):
    t = np.arange(float(n))
    u = np.stack([x0 + vx * t, y0 + vy * t, z0 + vz * t, np.full(n, vx), np.full(n, vy), np.full(n, vz)], axis=1)
    return tp.TraceSolution(t, u, "Success", "mock")


def test_detector_kats_on_gpu(tp):
    disk = tp.Disk(tp.Plane((0.0, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    area = math.pi * 25.0
    s1 = _line_sol(tp, -10.0, 0.0, 1.0, 0.0)
    s2 = _line_sol(tp, -10.0, 10.0, 1.0, 0.0)
    s3 = _line_sol(tp, 5.0, -10.0, 0.0, 1.0)
    nf, vf = tp.get_particle_flux(s1, disk)
    assert math.isclose(nf, 1.0 / area) and np.allclose(vf, [1.0 / area, 0, 0])
    vs, ws = tp.get_particle_crossings(s1, disk)
    assert len(vs) == 1 and ws.sum() == 1.0 and np.allclose(vs[0], [1.0, 0.0, 0.0])
    for s in (s2, s3):
        nf, vf = tp.get_particle_flux(s, disk)
        assert nf == 0.0 and np.all(vf == 0.0)
    nf, vf = tp.get_particle_fluxes([s1, s2, s3], disk, 1.0)
    assert math.isclose(nf, 1.0 / area)
    nf, _ = tp.get_particle_fluxes([s1, s2, s3], disk, [1.0, 2.0, 3.0])
    assert math.isclose(nf, 1.0 / area)
    nf, vf = tp.get_particle_fluxes([s1, s1, s2], disk, [1.0, 2.0, 3.0])
    assert math.isclose(nf, 3.0 / area) and np.allclose(vf, [3.0 / area, 0, 0])
    nf, vf = tp.get_particle_flux(s1, disk, 2.0)
    assert math.isclose(nf, 2.0 / area) and np.allclose(vf, [2.0 / area, 0, 0])
    vs, ws = tp.get_particle_crossings(s1, tp.Plane((0.0, 0.0, 0.0), (1.0, 0.0, 0.0)), 3.0)
    assert len(vs) == 1 and ws.sum() == 3.0 and np.allclose(vs[0], [1.0, 0, 0])
    nf, vf = tp.get_particle_flux(s1, tp.Sphere((0.0, 0.0, 0.0), 5.0))
    sa = 4 * math.pi * 25.0
    assert math.isclose(nf, 2.0 / sa) and np.allclose(vf, [2.0 / sa, 0, 0])
    sa_, sb_ = _line_sol(tp, -10.0, 0.0, 1.0, 0.0), _line_sol(tp, -10.0, 0.0, 2.0, 0.0)
    va, wa = tp.get_particle_crossings(sa_, disk, 2.0)
    vb, wb = tp.get_particle_crossings(sb_, disk, 1.0)
    assert va[0][0] == 1.0 and wa[0] == 2.0 and vb[0][0] == 2.0 and wb[0] == 1.0
    nfa, vfa = tp.get_particle_flux(sa_, disk, 2.0)
    nfb, vfb = tp.get_particle_flux(sb_, disk, 1.0)
    assert nfa == 2.0 / area and vfa[0] == 2.0 / area and nfb == 1.0 / area and vfb[0] == 2.0 / area
    # several detectors and ensembles
    one = tp.TraceSolution(np.array([0.0, 2.0]), np.array([[0.0, 0, 0, 1, 0, 0], [2.0, 0, 0, 1, 0, 0]]), "Success",
                           "mock")
    d1 = tp.Disk(tp.Plane((0.5, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    d2 = tp.Disk(tp.Plane((1.5, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    nfs, vfs = tp.get_particle_fluxes([one], [d1, d2], 1.0)
    assert np.allclose(nfs, [1.0 / area, 1.0 / area]) and np.allclose(vfs, [[1.0 / area, 0, 0]] * 2)
    d = tp.Disk(tp.Plane((1.0, 0.0, 0.0), (1.0, 0.0, 0.0)), 5.0)
    vs, ws = tp.get_particle_crossings([one, one], d, 2.5)
    assert len(vs) == 2 and np.all(ws == 2.5)
    vs, ws = tp.get_particle_crossings([one, one], [d, d], 4.0)
    assert len(vs) == 2 and len(vs[0]) == 2 and np.all(ws[0] == 4.0)
    # first crossing
    sz = _line_sol(tp, 0.0, 0.0, 0.0, 0.0, z0=-10.0, vz=1.0)
    st = tp.get_first_crossing(sz, tp.Plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0)))
    assert np.allclose(st, [0, 0, 0, 0, 0, 1.0])
    assert np.all(np.isnan(tp.get_first_crossing(sz, tp.Plane((0.0, 0.0, 20.0), (0.0, 0.0, 1.0)))))
    with pytest.raises(TypeError):
        tp.get_particle_flux(s1, tp.Plane((0.0, 0.0, 0.0), (1.0, 0.0, 0.0)))


def test_detectors_match_oracle_on_solutions(tp, orc):
    # gyrating protons drifting across detectors in crossed E, B fields
    rng = np.random.default_rng(4)
    n = 2048
    u0 = np.zeros((6, n))
    u0[:3] = rng.uniform(-2.0e5, 2.0e5, (3, n))
    u0[3:] = rng.normal(0.0, 1.0e5, (3, n))
    B0 = 1.0e-8
    T = tp.get_gyroperiod(B0)
    E = tp.UniformField((0.0, 5.0e-3, 0.0))
    prob = tp.TraceProblem(u0, (0.0, 20 * T), tp.prepare(E, tp.UniformField((0.0, 0.0, B0))))
    sols = tp.solve(prob, tp.Boris(), dt=T / 40, savestepinterval=2)
    surfs = [tp.Plane((0.0, 0.0, 0.0), (1.0, 0.2, 0.1)), tp.Disk(tp.Plane((1.0e5, 0.0, 0.0), (1.0, 0.0, 0.0)), 3.0e5),
             tp.Sphere((0.0, 0.0, 0.0), 2.5e5), tp.Disk(tp.Plane((0.0, 0.0, 1.0e5), (0.0, 0.0, 1.0)), 1.0e5)]
    w = rng.uniform(0.5, 2.0, n)
    sums, counts, rows, _ = orc.detect(sols.t_all, sols.u_all, sols.nsaved, surfs, weights=w)
    vs, ws = tp.get_particle_crossings(sols, surfs, w)
    k = 0
    for j in range(len(surfs)):
        assert len(ws[j]) == counts[j] and counts[j] > 0
        ref = rows[k:k + counts[j]]
        assert np.array_equal(ws[j], ref[:, 3])
        assert np.max(np.abs(vs[j] - ref[:, :3])) <= 1e-13 * np.max(np.abs(ref[:, :3]))
        k += counts[j]
    area = np.array([1.0] + [s.area() for s in surfs[1:]])
    nf, vf = tp.get_particle_fluxes(sols, surfs[1:], w)
    assert np.allclose(nf, sums[1:, 0] / area[1:], rtol=1e-12, atol=0)
    assert np.allclose(vf, sums[1:, 1:] / area[1:, None], rtol=1e-12, atol=1e-12 * np.abs(vf).max())
    for sf in surfs:
        _, _, _, first = orc.detect(sols.t_all, sols.u_all, sols.nsaved, [sf])
        got = tp.get_first_crossing(sols, sf)
        assert np.array_equal(np.isnan(got), np.isnan(first))
        ok = ~np.isnan(first)
        assert np.max(np.abs(got[ok] - first[ok])) <= 1e-13 * np.max(np.abs(first[ok]))
