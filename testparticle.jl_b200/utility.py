"""Scalar helpers of the reference's utility module used to set up problems.

Restated from src/utility/utility.jl (gyro helpers :148-270, energy2velocity
:327, sph2cart :50-56, get_perp_vector :119-126); host-side numpy.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import c, mi, qi


def get_gyrofrequency(B: float = 5.0e-9, q: float = qi, m: float = mi) -> float:
    """Gyrofrequency q B / m [rad/s]."""
    return q * B / m


def get_gyroperiod(B: float = 5.0e-9, q: float = qi, m: float = mi) -> float:
    """Gyroperiod 2 pi / omega [s]."""
    return 2 * math.pi / get_gyrofrequency(B, q, m)


def get_gyroradius(V: float, B: float, q: float = qi, m: float = mi) -> float:
    """Gyroradius V / omega [m]."""
    return V / get_gyrofrequency(B, q, m)


def energy2velocity(Ek, m: float = mi, q: float = qi):
    """Relativistic speed of a particle of kinetic energy Ek [eV]."""
    Ek = np.asarray(Ek, dtype=float)
    v = c * np.sqrt(1 - 1 / (1 + Ek * abs(q) / (m * c**2)) ** 2)
    return float(v) if v.ndim == 0 else v


def sph2cart(r, theta, phi):
    """(r, theta, phi) -> Cartesian vector, ((r sin(theta)) cos(phi), ...)."""
    st, ct = math.sin(theta), math.cos(theta)
    sp, cp = math.sin(phi), math.cos(phi)
    return np.array([r * st * cp, r * st * sp, r * ct])


def get_perp_vector(b):
    """Unit vectors e1, e2 with (e1, e2, b) right-handed and orthonormal."""
    b = np.asarray(b, dtype=float)
    bh = b / np.linalg.norm(b)
    v = np.array([0.0, 0.0, 1.0]) if abs(bh[2]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(v, bh)
    e1 = e1 / np.linalg.norm(e1)
    e2 = np.cross(bh, e1)
    return e1, e2
