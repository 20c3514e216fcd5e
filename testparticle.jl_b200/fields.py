"""Field descriptors the B200 library can evaluate on the device.

The reference accepts any Julia callable `F(x, t)` as a field (src/prepare.jl
:36-104).  A callable cannot cross a C ABI, so this package recognises the
field types that cover the reference's tests and workloads:

* ZeroField                                    src/utility/zero.jl:35-51
* UniformField(value)                          a constant vector
* AffineField(value, jac, rate)                value + jac @ x + rate * t
* DipoleField(moment, center, coef)            point dipole (Magnetostatics.Dipole)
* FieldInterpolator via build_interpolator     src/utility/interpolation.jl:217-235
  (order 1, uniform Cartesian grid, FillExtrap(NaN) / ClampExtrap() /
  PeriodicBC(endpoint=:exclusive) == WrapExtrap())

Any other callable raises NotImplementedError naming these types.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .constants import MU0_OVER_4PI


class AbstractField:
    """Base of the device-evaluable fields."""

    time_dependent = False

    def descriptor(self) -> _abi.FieldDesc:  # pragma: no cover - abstract
        raise NotImplementedError

    def keepalive(self):
        return None


class ZeroField(AbstractField):
    """Field that is identically zero."""

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_ZERO
        return d

    def __call__(self, x, t=0.0):
        return np.zeros(3)

    def __repr__(self):
        return "ZeroField()"


@dataclass
class UniformField(AbstractField):
    """F(x, t) = value."""

    value: tuple

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_UNIFORM
        for k in range(3):
            d.value[k] = float(self.value[k])
        return d

    def __call__(self, x, t=0.0):
        return np.asarray(self.value, dtype=float)


@dataclass
class AffineField(AbstractField):
    """F(x, t) = value + jac @ x + rate * t (jac[i][j] = dF_i/dx_j)."""

    value: tuple
    jac: tuple = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    rate: tuple = (0.0, 0.0, 0.0)

    @property
    def time_dependent(self):
        return any(float(r) != 0.0 for r in self.rate)

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_AFFINE
        J = np.asarray(self.jac, dtype=float).reshape(3, 3)
        for k in range(3):
            d.value[k] = float(self.value[k])
            d.rate[k] = float(self.rate[k])
        for k in range(9):
            d.jac[k] = float(J.flat[k])
        return d

    def __call__(self, x, t=0.0):
        J = np.asarray(self.jac, dtype=float).reshape(3, 3)
        return np.asarray(self.value, float) + J @ np.asarray(x, float) + np.asarray(self.rate, float) * t


@dataclass
class DipoleField(AbstractField):
    """Point dipole B = coef (3 (m.rhat) rhat - m) / |x - center|^3, coef = mu0/4pi."""

    moment: tuple
    center: tuple = (0.0, 0.0, 0.0)
    coef: float = MU0_OVER_4PI

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_DIPOLE
        for k in range(3):
            d.moment[k] = float(self.moment[k])
            d.center[k] = float(self.center[k])
        d.coef = float(self.coef)
        return d

    def __call__(self, x, t=0.0):
        d = np.asarray(x, float) - np.asarray(self.center, float)
        r = np.linalg.norm(d)
        rh = d / r
        m = np.asarray(self.moment, float)
        return self.coef * (3 * np.dot(m, rh) * rh - m) / r**3


# ---------------------------------------------------------------- grids
@dataclass(frozen=True)
class FillExtrap:
    """Outside the grid the field is `fill_value` (only NaN is supported)."""

    fill_value: float = math.nan


@dataclass(frozen=True)
class ClampExtrap:
    """Outside the grid the nearest boundary value is used."""


@dataclass(frozen=True)
class WrapExtrap:
    """Exclusive periodic wrapping with period L = n * dx."""


@dataclass(frozen=True)
class PeriodicBC:
    """PeriodicBC(endpoint='exclusive'), the same as WrapExtrap()."""

    endpoint: str = "exclusive"


def _bc_code(bc) -> int:
    if isinstance(bc, FillExtrap):
        if not (isinstance(bc.fill_value, float) and math.isnan(bc.fill_value)):
            raise NotImplementedError("FillExtrap supports NaN only")
        return _abi.TP_BC_FILL_NAN
    if isinstance(bc, ClampExtrap):
        return _abi.TP_BC_CLAMP
    if isinstance(bc, WrapExtrap):
        return _abi.TP_BC_PERIODIC
    if isinstance(bc, PeriodicBC):
        if bc.endpoint != "exclusive":
            raise NotImplementedError("PeriodicBC supports endpoint='exclusive' only")
        return _abi.TP_BC_PERIODIC
    raise TypeError(f"unknown boundary condition {bc!r}")


def _uniform_axis(g) -> tuple[float, float, int]:
    g = np.asarray(g, dtype=float)
    if g.ndim != 1 or g.size < 2:
        raise ValueError("grid axes must be 1-D with at least 2 nodes")
    if np.any(np.diff(g) <= 0):
        raise ValueError("grid vectors must be sorted (strictly increasing)")
    n = g.size
    dx = (g[-1] - g[0]) / (n - 1)
    if not np.allclose(np.diff(g), dx, rtol=1e-9, atol=0.0):
        raise NotImplementedError("only uniform (Cartesian) grids are supported on the B200")
    return float(g[0]), float(dx), int(n)


@dataclass
class FieldInterpolator(AbstractField):
    """Trilinear interpolator of a vector field on a uniform Cartesian grid.

    `data[c, i, j, k]` is component c at node (x[i], y[j], z[k]) -- the
    reference's (3, nx, ny, nz) array.  Stored column-major (Julia's memory
    order) so the device receives exactly the reference's layout.
    """

    data: np.ndarray
    origin: tuple
    spacing: tuple
    bc: object = field(default_factory=FillExtrap)

    def __post_init__(self):
        a = np.asarray(self.data)
        if a.ndim != 4 or a.shape[0] != 3:
            raise ValueError("Incompatible 3D force field and grid! (expected a (3, nx, ny, nz) array)")
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        self.data = np.asfortranarray(a)
        self._bc = _bc_code(self.bc)

    @property
    def n(self):
        return self.data.shape[1:]

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_GRID
        d.bc = self._bc
        d.dtype = _abi.TP_DTYPE_F32 if self.data.dtype == np.float32 else _abi.TP_DTYPE_F64
        for k in range(3):
            d.n[k] = int(self.data.shape[1 + k])
            d.origin[k] = float(self.origin[k])
            d.spacing[k] = float(self.spacing[k])
        d.data = self.data.ctypes.data_as(C.c_void_p)
        return d

    def keepalive(self):
        return self.data


def build_interpolator(A, x, y, z, order: int = 1, bc=None, gridtype="CartesianGrid"):
    """build_interpolator(CartesianGrid, A, x, y, z, order, bc) of the reference.

    Only order 1 (trilinear) on uniform Cartesian grids is evaluated on the
    device; other orders and grid types raise NotImplementedError.
    """
    if gridtype not in ("CartesianGrid", None):
        raise NotImplementedError(f"{gridtype} grids are not supported on the B200")
    if order not in (0, 1, 3):
        raise ValueError(f"Interpolation order {order} is not supported. Supported orders are 0, 1, and 3.")
    if order != 1:
        raise NotImplementedError("only order=1 (trilinear) interpolation runs on the B200")
    ax = [_uniform_axis(g) for g in (x, y, z)]
    A = np.asarray(A)
    if A.shape[1:] != tuple(a[2] for a in ax):
        raise ValueError("field array shape does not match the grid")
    return FieldInterpolator(A, tuple(a[0] for a in ax), tuple(a[1] for a in ax),
                             bc if bc is not None else FillExtrap())


def as_field(f) -> AbstractField:
    """Normalise a user field argument to a device-evaluable field."""
    if isinstance(f, AbstractField):
        return f
    if f is None:
        return ZeroField()
    if isinstance(f, (tuple, list, np.ndarray)) and np.asarray(f).shape == (3,):
        return UniformField(tuple(float(v) for v in f))
    raise NotImplementedError(
        "field not supported by EnsembleB200: use ZeroField, UniformField, AffineField, "
        "DipoleField or build_interpolator (Python/Julia callables cannot run on the device)")
