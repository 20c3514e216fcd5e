"""Virtual detectors: surface crossings and particle fluxes of solutions.

Mirrors the Meshes extension of the reference (ext/TestParticleMeshesExt.jl:
98-491): `Plane(point, normal)`, `Disk(plane, radius)` and
`Sphere(center, radius)` surfaces; `get_particle_crossings`,
`get_particle_flux`, `get_particle_fluxes` and `get_first_crossing`.  The
crossings are found on the device (tp_detect_*) over the packed saves of an
EnsembleSolution (or of solutions packed on the fly).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from .runtime import Context, _check, _ptr
from .solution import EnsembleSolution, TraceSolution


@dataclass(frozen=True)
class Plane:
    """Plane through `point` with normal `normal` (normalised, as Meshes' normal(plane))."""

    point: tuple
    normal: tuple

    def descriptor(self) -> _abi.Surface:
        d = _abi.Surface()
        d.kind = _abi.TP_SURF_PLANE
        nv = np.asarray(self.normal, dtype=float)
        nv = nv / np.linalg.norm(nv)
        for k in range(3):
            d.point[k] = float(self.point[k])
            d.normal[k] = float(nv[k])
        return d


@dataclass(frozen=True)
class Disk:
    """Disk of `radius` centred at the plane's point."""

    plane: Plane
    radius: float

    def descriptor(self) -> _abi.Surface:
        d = self.plane.descriptor()
        d.kind = _abi.TP_SURF_DISK
        d.radius = float(self.radius)
        return d

    def area(self) -> float:
        return math.pi * (self.radius * self.radius)


@dataclass(frozen=True)
class Sphere:
    center: tuple
    radius: float

    def descriptor(self) -> _abi.Surface:
        d = _abi.Surface()
        d.kind = _abi.TP_SURF_SPHERE
        for k in range(3):
            d.point[k] = float(self.center[k])
        d.radius = float(self.radius)
        return d

    def area(self) -> float:
        return (4.0 * math.pi) * (self.radius * self.radius)


def _packed(sols):
    """(t, u, nsaved) of one solution, an EnsembleSolution or a sequence of solutions."""
    if isinstance(sols, EnsembleSolution):
        return sols.t_all, sols.u_all, sols.nsaved
    if isinstance(sols, TraceSolution):
        sols = [sols]
    sols = list(sols)
    t = np.concatenate([np.asarray(s.t, dtype=float) for s in sols])
    u = np.concatenate([np.asarray(s.u, dtype=float).reshape(len(s.t), -1) for s in sols])
    ns = np.array([len(s.t) for s in sols], dtype=np.int32)
    return t, u, ns


def _weights(weights, n):
    if np.ndim(weights) == 0:
        return None, float(weights)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    if w.size != n:
        raise ValueError("one weight per trajectory")
    return w, 1.0


def _surfaces(surface):
    many = isinstance(surface, (list, tuple))
    surfs = list(surface) if many else [surface]
    for sf in surfs:
        if not isinstance(sf, (Plane, Disk, Sphere)):
            raise TypeError("surfaces are Plane, Disk or Sphere")
    return surfs, many


def _call_crossings(sols, surface, weights, device):
    t, u, ns = _packed(sols)
    t, u, ns = (np.ascontiguousarray(t, dtype=np.float64), np.ascontiguousarray(u, dtype=np.float64),
                np.ascontiguousarray(ns, dtype=np.int32))
    surfs, many = _surfaces(surface)
    w, w0 = _weights(weights, ns.size)
    descs = (_abi.Surface * len(surfs))(*[sf.descriptor() for sf in surfs])
    ctx = Context.get(device)
    counts = np.zeros(len(surfs), dtype=np.int64)
    args = (ctx.handle, _ptr(t), _ptr(u), u.shape[1], _ptr(ns), ns.size, descs, len(surfs), _ptr(w), w0)
    _check(ctx.lib, ctx.handle, ctx.lib.tp_detect_crossings(*args, _ptr(counts), None), "tp_detect_crossings")
    rows = np.empty((int(counts.sum()), 4))
    _check(ctx.lib, ctx.handle, ctx.lib.tp_detect_crossings(*args, _ptr(counts), _ptr(rows)), "tp_detect_crossings")
    out_v, out_w, k = [], [], 0
    for c in counts:
        out_v.append(rows[k:k + c, :3])
        out_w.append(rows[k:k + c, 3])
        k += int(c)
    return (out_v, out_w) if many else (out_v[0], out_w[0])


def get_particle_crossings(sols, surface, weights=1.0, device: int = 0):
    """Crossing velocities (k, 3) and weights (k,) -- lists of them for a list of surfaces."""
    return _call_crossings(sols, surface, weights, device)


def get_particle_fluxes(sols, surface, weights=1.0, device: int = 0):
    """(number flux density, velocity flux density) through disks / spheres:
    sums of weights and of weight * velocity over all crossings, divided by the area."""
    t, u, ns = _packed(sols)
    t, u, ns = (np.ascontiguousarray(t, dtype=np.float64), np.ascontiguousarray(u, dtype=np.float64),
                np.ascontiguousarray(ns, dtype=np.int32))
    surfs, many = _surfaces(surface)
    if any(isinstance(sf, Plane) for sf in surfs):
        raise TypeError("fluxes need a Disk or a Sphere (a surface with an area)")
    w, w0 = _weights(weights, ns.size)
    descs = (_abi.Surface * len(surfs))(*[sf.descriptor() for sf in surfs])
    ctx = Context.get(device)
    nf = np.empty(len(surfs))
    vf = np.empty((len(surfs), 3))
    code = ctx.lib.tp_detect_fluxes(ctx.handle, _ptr(t), _ptr(u), u.shape[1], _ptr(ns), ns.size, descs, len(surfs),
                                    _ptr(w), w0, _ptr(nf), _ptr(vf))
    _check(ctx.lib, ctx.handle, code, "tp_detect_fluxes")
    return (nf, vf) if many else (float(nf[0]), vf[0])


def get_particle_flux(sol, surface, weight: float = 1.0, device: int = 0):
    """get_particle_fluxes of one solution and one disk / sphere."""
    return get_particle_fluxes(sol, surface, weight, device)


def get_first_crossing(sols, surface, device: int = 0):
    """The state (6 values) at each trajectory's first crossing of `surface`, NaN if none;
    (6,) for one solution, (n, 6) otherwise."""
    t, u, ns = _packed(sols)
    t, u, ns = (np.ascontiguousarray(t, dtype=np.float64), np.ascontiguousarray(u, dtype=np.float64),
                np.ascontiguousarray(ns, dtype=np.int32))
    if not isinstance(surface, (Plane, Disk, Sphere)):
        raise TypeError("surfaces are Plane, Disk or Sphere")
    desc = surface.descriptor()
    out = np.empty((ns.size, 6))
    ctx = Context.get(device)
    code = ctx.lib.tp_detect_first_crossing(ctx.handle, _ptr(t), _ptr(u), u.shape[1], _ptr(ns), ns.size,
                                            C.byref(desc), _ptr(out))
    _check(ctx.lib, ctx.handle, code, "tp_detect_first_crossing")
    return out[0] if isinstance(sols, TraceSolution) else out
