"""Seeded synthetic inputs of the five benchmark configurations.

No dataset is involved: every input is drawn from a counter-based SplitMix64
stream (Steele, Lea & Flood 2014; the mixer also used by the reference's
_rng_seed, src/utility/utility.jl:36-42) with seed 20261203 + config, so the
tables are identical on every machine and numpy version.  Normals use the
Box-Muller transform.  "Maxwellian with thermal speed v_th" means each
velocity component is N(0, v_th / sqrt(2)) (get_thermal_speed = sqrt(2p/(nm)),
src/sampler.jl:56).

config 1  1000 protons, uniform B = 1e-8 z, 1e4 Boris steps (CPU-runnable)
config 2  1e6 protons in a 128^3 periodic turbulent field, 1e4 steps
config 3  1e6 protons in the Earth dipole, MultistepBoris4(n=2) / AdaptiveBoris
config 4  2^20 guiding centres (half e-, half p+) in the dipole, RK4 / RK45
config 5  adjoint of Boris in the config-2 field (2^18 protons, 4096 steps)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .constants import BMoment_Earth, Electron, MU0_OVER_4PI, Proton, Re, eV, mi, qi
from .fields import DipoleField, FieldInterpolator, UniformField, WrapExtrap, ZeroField
from .utility import get_gyroperiod

SEED0 = 20261203
_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class SplitMix64:
    """Counter-based SplitMix64: value k of the stream is mix(seed + (k+1) * gamma)."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed % (1 << 64))
        self.k = 0

    def next_u64(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            idx = np.arange(self.k + 1, self.k + n + 1, dtype=np.uint64)
            z = self.seed + idx * _GAMMA
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        self.k += n
        return z

    def uniform(self, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (self.next_u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def normal(self, n: int, sigma: float = 1.0) -> np.ndarray:
        u1 = 1.0 - self.uniform(n)  # (0, 1]
        u2 = self.uniform(n)
        return sigma * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def dipole_B(r: np.ndarray, moment=BMoment_Earth, coef=MU0_OVER_4PI) -> np.ndarray:
    """Dipole field at rows of r (N, 3), float64."""
    m = np.asarray(moment, dtype=float)
    d = np.linalg.norm(r, axis=1, keepdims=True)
    rh = r / d
    return coef * (3 * (rh @ m)[:, None] * rh - m) / d**3


@dataclass
class FullOrbitWorkload:
    name: str
    u0: np.ndarray            # (6, N)
    tspan: tuple
    dt: object                # float or (N,) array
    E: object
    B: object
    savestepinterval: int
    species: object = Proton
    tend: object = None       # optional (N,) per-particle tspan[2]
    isoutside: object = None
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.u0.shape[1]

    @property
    def nt(self) -> int:
        dt = np.asarray(self.dt)
        if self.tend is not None:
            return int(np.rint(np.max(np.abs((np.asarray(self.tend) - self.tspan[0]) / dt))))
        return int(np.rint(abs((self.tspan[1] - self.tspan[0]) / float(np.max(dt)))))


# ------------------------------------------------------------------ config 1
def config1(n: int = 1000) -> FullOrbitWorkload:
    rng = SplitMix64(SEED0 + 1)
    B0 = 1.0e-8
    dt = get_gyroperiod(B0) / 100
    u0 = np.empty((6, n))
    u0[0:3] = rng.uniform(3 * n, -1.0, 1.0).reshape(3, n)
    u0[3:6] = rng.normal(3 * n, 1.0e5 / math.sqrt(2)).reshape(3, n)
    return FullOrbitWorkload("config1_plain_boris_uniform_B", u0, (0.0, 1.0e4 * dt), dt, ZeroField(),
                             UniformField((0.0, 0.0, B0)), 100)


# ------------------------------------------------------------------ config 2
def turbulent_grid(nx: int = 128, dx: float = 1.0e5, B0: float = 5.0e-9, nmodes: int = 64,
                   rms_frac: float = 0.3, u=(4.0e5, 0.0, 0.0), seed: int = SEED0 + 2):
    """E and B node arrays (3, nx, nx, nx) float32 of the config-2 field.

    B = B0 z + sum_j A_j e_j cos(k_j . x + phi_j): |k_j| log-spaced in
    [2 pi/L, 16 pi/L], isotropic directions snapped to the integer lattice
    (2 pi / L) Z^3 (exactly periodic), e_j perpendicular to k_j (div B = 0),
    A_j ~ |k_j|^(-1/3), RMS |dB| = rms_frac * B0 over the grid.  E = -u x B.
    """
    rng = SplitMix64(seed)
    L = nx * dx
    kmag = np.exp(np.linspace(math.log(1.0), math.log(8.0), nmodes))  # in units of 2 pi / L
    kint = np.zeros((nmodes, 3), dtype=np.int64)
    for j in range(nmodes):
        while True:
            cz = rng.uniform(1, -1.0, 1.0)[0]
            ph = rng.uniform(1, 0.0, 2 * math.pi)[0]
            s = math.sqrt(max(0.0, 1 - cz * cz))
            dvec = np.array([s * math.cos(ph), s * math.sin(ph), cz])
            k = np.rint(kmag[j] * dvec).astype(np.int64)
            if np.any(k != 0):
                kint[j] = k
                break
    amps = np.empty(nmodes)
    pols = np.empty((nmodes, 3))
    phases = rng.uniform(nmodes, 0.0, 2 * math.pi)
    for j in range(nmodes):
        kv = kint[j].astype(float)
        kh = kv / np.linalg.norm(kv)
        a = np.array([1.0, 0.0, 0.0]) if abs(kh[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        e1 = np.cross(kh, a)
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(kh, e1)
        psi = rng.uniform(1, 0.0, 2 * math.pi)[0]
        pols[j] = math.cos(psi) * e1 + math.sin(psi) * e2
        amps[j] = np.linalg.norm(kv) ** (-1.0 / 3.0)
    idx = np.arange(nx)
    dB = np.zeros((3, nx, nx, nx))
    for j in range(nmodes):
        w = 2 * math.pi / nx
        ex = np.exp(1j * w * kint[j, 0] * idx)
        ey = np.exp(1j * w * kint[j, 1] * idx)
        ez = np.exp(1j * w * kint[j, 2] * idx)
        ph = np.exp(1j * phases[j]) * ex[:, None, None] * ey[None, :, None] * ez[None, None, :]
        c = ph.real
        for comp in range(3):
            dB[comp] += amps[j] * pols[j, comp] * c
    rms = math.sqrt(np.mean(np.sum(dB**2, axis=0)))
    dB *= rms_frac * B0 / rms
    B = dB
    B[2] += B0
    ux, uy, uz = u
    E = np.empty_like(B)
    E[0] = -(uy * B[2] - uz * B[1])
    E[1] = -(uz * B[0] - ux * B[2])
    E[2] = -(ux * B[1] - uy * B[0])
    return E.astype(np.float32), B.astype(np.float32), L


def config2(n: int = 1_000_000, nx: int = 128, nt: int = 10_000, ssi: int = 1000) -> FullOrbitWorkload:
    dx = 1.0e5
    B0 = 5.0e-9
    Ea, Ba, L = turbulent_grid(nx, dx, B0)
    E = FieldInterpolator(Ea, (0.0, 0.0, 0.0), (dx, dx, dx), WrapExtrap())
    B = FieldInterpolator(Ba, (0.0, 0.0, 0.0), (dx, dx, dx), WrapExtrap())
    rng = SplitMix64(SEED0 + 102)
    u0 = np.empty((6, n))
    u0[0:3] = rng.uniform(3 * n, 0.0, L).reshape(3, n)
    u0[3:6] = rng.normal(3 * n, 2.0e5 / math.sqrt(2)).reshape(3, n)
    dt = get_gyroperiod(B0) / 50
    return FullOrbitWorkload("config2_gridded_boris_128cube", u0, (0.0, nt * dt), dt, E, B, ssi,
                             extra={"L": L, "B0": B0})


# ------------------------------------------------------------------ config 3
def config3(n: int = 1_000_000, nt: int = 10_000, ssi: int = 1000) -> FullOrbitWorkload:
    """Dipole ensemble; dt_i = 0.02 T_gyro(|B(r0)|), tspan_i = nt * dt_i."""
    rng = SplitMix64(SEED0 + 3)
    m = np.array([0.0, 0.0, -8.0e22])
    Ek = np.exp(rng.uniform(n, math.log(1.0e4), math.log(1.0e7)))  # eV
    v = np.sqrt(2 * Ek * eV / mi)
    cos_a = rng.uniform(n, -1.0, 1.0)
    Lsh = rng.uniform(n, 3.0, 7.0)
    phi = rng.uniform(n, 0.0, 2 * math.pi)
    psi = rng.uniform(n, 0.0, 2 * math.pi)
    r = np.stack([Lsh * Re * np.cos(phi), Lsh * Re * np.sin(phi), np.zeros(n)], axis=1)
    B = dipole_B(r, m)
    Bm = np.linalg.norm(B, axis=1)
    bh = B / Bm[:, None]
    # get_perp_vector (utility.jl:119-126) row-wise: |bh_z| ~ 1 at the equator -> v = y
    vref = np.where(np.abs(bh[:, 2:3]) < 0.9, np.array([0.0, 0.0, 1.0]), np.array([0.0, 1.0, 0.0]))
    e1 = np.cross(vref, bh)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    e2 = np.cross(bh, e1)
    sin_a = np.sqrt(1 - cos_a**2)
    vel = v[:, None] * (cos_a[:, None] * bh + sin_a[:, None] * (np.cos(psi)[:, None] * e1 +
                                                                 np.sin(psi)[:, None] * e2))
    u0 = np.concatenate([r, vel], axis=1).T.copy()
    Tg = 2 * math.pi * mi / (qi * Bm)
    dt = 0.02 * Tg
    from .problems import TerminateShell
    return FullOrbitWorkload("config3_dipole_ensemble", u0, (0.0, float(nt * dt.max())), dt, ZeroField(),
                             DipoleField(tuple(m)), ssi, tend=nt * dt,
                             isoutside=TerminateShell(Re, 15 * Re), extra={"Ek_eV": Ek})


# ------------------------------------------------------------------ config 4
@dataclass
class GCWorkload:
    name: str
    y0: np.ndarray       # (4, N)
    q: np.ndarray
    q2m: np.ndarray
    mu: np.ndarray
    m: np.ndarray
    E: object
    B: object
    tau_b: np.ndarray    # bounce periods
    extra: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.y0.shape[1]


def config4(n: int = 1 << 20) -> GCWorkload:
    """Guiding centres in the dipole; half electrons (first half), half protons."""
    rng = SplitMix64(SEED0 + 4)
    mvec = np.array([0.0, 0.0, -8.0e22])
    half = n // 2
    mass = np.where(np.arange(n) < half, Electron.m, Proton.m)
    charge = np.where(np.arange(n) < half, Electron.q, Proton.q)
    Ek = np.exp(rng.uniform(n, math.log(1.0e3), math.log(1.0e6)))
    c = 299792458.0  # relativistic speed (energy2velocity, utility.jl:327): 1 MeV electrons
    v = c * np.sqrt(1 - 1 / (1 + Ek * np.abs(charge) / (mass * c**2)) ** 2)
    alpha = np.deg2rad(rng.uniform(n, 10.0, 90.0))
    Lsh = rng.uniform(n, 2.0, 8.0)
    phi = rng.uniform(n, 0.0, 2 * math.pi)
    X = np.stack([Lsh * Re * np.cos(phi), Lsh * Re * np.sin(phi), np.zeros(n)], axis=1)
    Beq = np.linalg.norm(dipole_B(X, mvec), axis=1)
    vpar = v * np.cos(alpha)
    mu = mass * (v * np.sin(alpha)) ** 2 / (2 * Beq)
    tau_b = 4 * Lsh * Re / v * (1.30 - 0.56 * np.sin(alpha))
    y0 = np.concatenate([X, vpar[:, None]], axis=1).T.copy()
    return GCWorkload("config4_gc_dipole", y0, charge, charge / mass, mu, mass, ZeroField(),
                      DipoleField(tuple(mvec)), tau_b)


# ------------------------------------------------------------------ config 5
def config5(n: int = 1 << 18, nt: int = 4096, nx: int = 128) -> FullOrbitWorkload:
    """Adjoint workload: protons drawn as in config 2 (same field), nt steps.

    extra["target_offset"] (N, 3) holds the seeded N(0, (1e5 m)^2) offsets of
    the targets x_target = x_N(float64 solve) + offset; the loss is
    mean_i |x_N,i - x_target,i|^2.
    """
    w = config2(n=n, nx=nx, nt=nt, ssi=nt)
    rng = SplitMix64(SEED0 + 5)
    w.name = "config5_boris_adjoint_128cube"
    w.extra["target_offset"] = rng.normal(3 * n, 1.0e5).reshape(n, 3)
    return w


def loss_and_grad(x_final: np.ndarray, x_target: np.ndarray):
    """L = mean_i |x_i - t_i|^2 and dL/d(final state) (N, 6; zero velocity part)."""
    d = x_final[:, :3] - x_target
    n = d.shape[0]
    g = np.zeros((n, 6))
    g[:, :3] = 2.0 * d / n
    return float(np.sum(d * d) / n), g
