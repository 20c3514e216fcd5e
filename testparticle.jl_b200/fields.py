"""Field descriptors the B200 library can evaluate on the device.

The reference accepts any Julia callable `F(x, t)` as a field (src/prepare.jl
:36-104).  A callable cannot cross a C ABI, so this package recognises the
field types that cover the reference's tests and workloads:

* ZeroField                                    src/utility/zero.jl:35-51
* UniformField(value)                          a constant vector
* AffineField(value, jac, rate)                value + jac @ x + rate * t
* DipoleField(moment, center, coef)            point dipole (Magnetostatics.Dipole)
* FieldInterpolator via build_interpolator     src/utility/interpolation.jl:15-311
  (orders 0 / 1 / 3; Cartesian, rectilinear and spherical grids; 1-D, 2-D
  and 3-D interpolants; FillExtrap(NaN) / ClampExtrap() / PeriodicBC)

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
class QuadraticField(AbstractField):
    """F_i(x, t) = value_i + sum_j jac_ij x_j + sum_jk quad_ijk x_j x_k + rate_i t.

    Covers the reference's quadratic test fields, e.g. the magnetic bottle
    B = B0 (-a x z, -a y z, 1 + a z^2) of test/test_hybrid.jl:61-68
    (see QuadraticField.bottle).
    """

    value: tuple
    jac: tuple = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    quad: object = None          # (3, 3, 3): quad[i][j][k] multiplies x_j x_k in F_i
    rate: tuple = (0.0, 0.0, 0.0)

    @classmethod
    def bottle(cls, B0: float, alpha: float) -> "QuadraticField":
        Q = np.zeros((3, 3, 3))
        Q[0, 0, 2] = -B0 * alpha
        Q[1, 1, 2] = -B0 * alpha
        Q[2, 2, 2] = B0 * alpha
        return cls((0.0, 0.0, B0), quad=Q)

    @property
    def time_dependent(self):
        return any(float(r) != 0.0 for r in self.rate)

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_QUADRATIC
        J = np.asarray(self.jac, dtype=float).reshape(3, 3)
        Q = np.zeros(27) if self.quad is None else np.asarray(self.quad, dtype=float).reshape(27)
        for k in range(3):
            d.value[k] = float(self.value[k])
            d.rate[k] = float(self.rate[k])
        for k in range(9):
            d.jac[k] = float(J.flat[k])
        for k in range(27):
            d.quad[k] = float(Q[k])
        return d

    def __call__(self, x, t=0.0):
        x = np.asarray(x, float)
        J = np.asarray(self.jac, dtype=float).reshape(3, 3)
        Q = np.zeros((3, 3, 3)) if self.quad is None else np.asarray(self.quad, dtype=float).reshape(3, 3, 3)
        return (np.asarray(self.value, float) + J @ x + np.einsum("ijk,j,k->i", Q, x, x)
                + np.asarray(self.rate, float) * t)


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
    """PeriodicBC(endpoint='exclusive') (period n * dx, the same as
    WrapExtrap()) or endpoint='inclusive' (period (n - 1) * dx: the last node
    repeats the first)."""

    endpoint: str = "exclusive"


class CartesianGrid:
    """Grid-type marker of build_interpolator (Meshes.CartesianGrid)."""


class RectilinearGrid:
    """Grid-type marker: axes given by node coordinates (Meshes.RectilinearGrid)."""


class StructuredGrid:
    """Grid-type marker: spherical (r, theta, phi) axes (Meshes.StructuredGrid)."""


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
        if bc.endpoint == "exclusive":
            return _abi.TP_BC_PERIODIC
        if bc.endpoint == "inclusive":
            return _abi.TP_BC_PERIODIC_INCLUSIVE
        raise ValueError(f"unknown PeriodicBC endpoint {bc.endpoint!r}")
    raise TypeError(f"unknown boundary condition {bc!r}")


_ORDER = {0: _abi.TP_ORDER_CONSTANT, 1: _abi.TP_ORDER_LINEAR, 3: _abi.TP_ORDER_CUBIC}


def _axis(g, force_coords: bool = False):
    """(origin, spacing, n, coords): coords is None for a uniform axis."""
    g = np.asarray(g, dtype=float)
    if g.ndim != 1 or g.size < 2:
        raise ValueError("grid axes must be 1-D with at least 2 nodes")
    if np.any(np.diff(g) <= 0):
        raise ValueError("grid vectors must be sorted (strictly increasing)")
    n = g.size
    dx = (g[-1] - g[0]) / (n - 1)
    if not force_coords and np.allclose(np.diff(g), dx, rtol=1e-9, atol=0.0):
        return float(g[0]), float(dx), int(n), None
    return float(g[0]), float(dx), int(n), np.ascontiguousarray(g)


@dataclass
class FieldInterpolator(AbstractField):
    """A gridded vector field: the reference's FieldInterpolator /
    FieldInterpolator2D / FieldInterpolator1D / SphericalFieldInterpolator
    (src/utility/interpolation.jl:15-117).

    `data[c, i, j, k]` is component c at node (i, j, k) -- the reference's
    (3, n1, n2, n3) array -- stored column-major (Julia's memory order) so the
    device receives exactly the reference's layout.  Unused axes of 1-D / 2-D
    interpolants have one node.  `axes[a]` holds the node coordinates of a
    non-uniform axis (None: origin + k * spacing).  Scalar grids are carried
    as the first component of a vector field.
    """

    data: np.ndarray
    origin: tuple
    spacing: tuple
    bc: object = field(default_factory=FillExtrap)
    order: int = 1
    geometry: str = "cartesian"      # "spherical", or "spherical_scalar" for a scalar
    ndim: int = 3
    dir: int = 0                     # 1-D: the coordinate read (0-based)
    axes: tuple = (None, None, None)

    def __post_init__(self):
        a = np.asarray(self.data)
        if a.ndim == 4 - (3 - self.ndim) and a.shape[0] == 3 and self.ndim < 3:
            a = a.reshape(a.shape + (1,) * (4 - a.ndim))
        if a.ndim != 4 or a.shape[0] != 3:
            raise ValueError("Incompatible 3D force field and grid! (expected a (3, nx, ny, nz) array)")
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        self.data = np.asfortranarray(a)
        self._bc = _bc_code(self.bc)
        if self.order not in _ORDER:
            raise ValueError(f"Interpolation order {self.order} is not supported. "
                             "Supported orders are 0, 1, and 3.")
        self._axes = tuple(None if c is None else np.ascontiguousarray(c, dtype=np.float64) for c in self.axes)

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
            c = self._axes[k]
            d.axis[k] = None if c is None else c.ctypes.data
        d.data = self.data.ctypes.data_as(C.c_void_p)
        d.order = _ORDER[self.order]
        d.geometry = {"cartesian": _abi.TP_GRID_CARTESIAN, "spherical": _abi.TP_GRID_SPHERICAL,
                      "spherical_scalar": _abi.TP_GRID_SPHERICAL_SCALAR}[self.geometry]
        d.ndim = int(self.ndim)
        d.dir = int(self.dir)
        return d

    def keepalive(self):
        return (self.data, self._axes)


def _vector_data(A, ngrid: int) -> np.ndarray:
    """(3, n...) vector data, or a scalar (n...) array carried as component 0."""
    A = np.asarray(A)
    if A.ndim == ngrid + 1 and A.shape[0] == 3:
        return A
    if A.ndim == ngrid:
        V = np.zeros((3,) + A.shape, dtype=A.dtype if A.dtype in (np.float32, np.float64) else np.float64)
        V[0] = A
        return V
    raise ValueError(f"Incompatible {ngrid}D force field and grid!")


def build_interpolator(*args, dir: int = 1, coeffs=None):
    """build_interpolator([gridtype,] A, grids..., order=1, bc=FillExtrap(NaN); dir, coeffs).

    The reference's entry point (src/utility/interpolation.jl:190-311):
    `gridtype` is CartesianGrid (default; 1, 2 or 3 axes, uniform or given by
    node coordinates), RectilinearGrid (order 1 only) or StructuredGrid
    (spherical r, theta, phi: r and theta fill NaN outside, phi periodic).
    `order` is 0, 1 or 3 (cubic on uniform axes).  `dir` (1-based) selects the
    coordinate a 1-D interpolant reads.  `coeffs` is accepted for signature
    compatibility (the cubic is always evaluated on the fly).
    """
    args = list(args)
    gridtype = CartesianGrid
    if args and isinstance(args[0], type) and args[0] in (CartesianGrid, RectilinearGrid, StructuredGrid):
        gridtype = args.pop(0)
    elif args and isinstance(args[0], str):
        gridtype = {"CartesianGrid": CartesianGrid, "RectilinearGrid": RectilinearGrid,
                    "StructuredGrid": StructuredGrid}[args.pop(0)]
    if not args:
        raise TypeError("build_interpolator needs a field array")
    A = args.pop(0)
    grids = []
    while args and not isinstance(args[0], (int, np.integer)) and not isinstance(
            args[0], (FillExtrap, ClampExtrap, WrapExtrap, PeriodicBC)) and args[0] is not None:
        grids.append(args.pop(0))
    order = int(args.pop(0)) if args and args[0] is not None else 1
    if args and args[0] is None:
        args.pop(0)
    bc = args.pop(0) if args else None
    if args:
        raise TypeError("too many arguments to build_interpolator")
    if order not in _ORDER:
        raise ValueError(f"Interpolation order {order} is not supported. Supported orders are 0, 1, and 3.")
    if not 1 <= len(grids) <= 3:
        raise ValueError("build_interpolator takes 1, 2 or 3 grid axes")
    bc = bc if bc is not None else FillExtrap()
    if gridtype is StructuredGrid:
        if len(grids) != 3:
            raise ValueError("StructuredGrid needs r, theta and phi axes")
        ax = [_axis(grids[0]), _axis(grids[1]), _axis(grids[2])]
        if ax[2][3] is not None:
            raise NotImplementedError("the phi axis of a spherical grid must be uniform")
        r0 = ax[0][0]
        t0, t1 = ax[1][0], ax[1][0] + ax[1][1] * (ax[1][2] - 1)
        p0, p1 = ax[2][0], ax[2][0] + ax[2][1] * (ax[2][2] - 1)
        if r0 < 0:
            raise ValueError("r must be non-negative.")
        if t0 < -1e-12 or t1 > math.pi + 1e-12:
            raise ValueError("θ must be within [0, π].")
        if p0 < -1e-12 or p1 > 2 * math.pi + 1e-12:
            raise ValueError("ϕ must be within [0, 2π].")
        data = _vector_data(A, 3)
        geometry = "spherical" if np.ndim(A) == 4 else "spherical_scalar"
        ndim = 3
    else:
        rect = gridtype is RectilinearGrid
        if rect and order != 1:
            raise ValueError("RectilinearGrid (CartesianNonUniform) only supports order=1 (Linear) interpolation.")
        ax = [_axis(g, force_coords=rect) for g in grids]
        if order == 3 and any(a[3] is not None for a in ax):
            raise NotImplementedError("cubic interpolation runs on uniform axes")
        ndim = len(grids)
        data = _vector_data(A, ndim)
        geometry = "cartesian"
        while len(ax) < 3:
            ax.append((0.0, 1.0, 1, None))
    if tuple(data.shape[1:1 + len(grids)]) != tuple(a[2] for a in ax[:len(grids)]):
        raise ValueError("field array shape does not match the grid")
    return FieldInterpolator(data, tuple(a[0] for a in ax), tuple(a[1] for a in ax), bc, order=order,
                             geometry=geometry, ndim=ndim, dir=int(dir) - 1 if ndim == 1 else 0,
                             axes=tuple(a[3] for a in ax))


class LazyTimeInterpolator(AbstractField):
    """LazyTimeInterpolator(times, loader) (src/utility/interpolation.jl:337-430).

    `loader(i)` (1-based, as in the reference) returns the field at times[i];
    the field at time t blends the two snapshots around t linearly and is
    clamped to the first / last snapshot outside the times.  The reference
    loads snapshots on demand and keeps two; here every snapshot is loaded
    once and stays resident on the device (HBM holds hundreds of 128^3 grids).
    """

    time_dependent = True

    def __init__(self, times, loader):
        self.times = np.ascontiguousarray(np.asarray(times, dtype=np.float64).reshape(-1))
        if self.times.size < 1:
            raise ValueError("LazyTimeInterpolator needs at least one time")
        if np.any(np.diff(self.times) < 0):
            raise ValueError("times must be sorted")
        self.snapshots = [as_field(loader(i + 1)) for i in range(self.times.size)]
        if any(isinstance(f, LazyTimeInterpolator) for f in self.snapshots):
            raise ValueError("a snapshot cannot be a LazyTimeInterpolator")

    def descriptor(self):
        descs = [f.descriptor() for f in self.snapshots]
        arr = (_abi.FieldDesc * len(descs))(*descs)
        self._arr = arr  # the descriptor array must outlive the upload
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_SERIES
        d.nseries = len(descs)
        d.series_times = self.times.ctypes.data
        d.series = C.cast(arr, C.c_void_p).value
        return d

    def keepalive(self):
        return (self.times, getattr(self, "_arr", None), [f.keepalive() for f in self.snapshots])


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
