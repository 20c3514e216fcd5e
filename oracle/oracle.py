"""ctypes wrapper of liboracle.so, the CPU restatement of the reference solver.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py to check and to time the CUDA library.  The
product never imports it.

Descriptors are the library's own (include/tp_abi.h via the package's _abi
module), so the same run description drives both.  Fields and the
termination predicate may also be Python callables (the reference tests'
closures), passed as C callbacks.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

FIELD_CB = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_void_p)
JAC_CB = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_void_p)
OUT_CB = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_void_p)


class FieldCB(C.Structure):
    _fields_ = [("f", FIELD_CB), ("j", JAC_CB), ("user", C.c_void_p)]


class TermCB(C.Structure):
    _fields_ = [("f", OUT_CB), ("user", C.c_void_p)]


_lib = None


def build() -> Path:
    """Compile liboracle.so with its Makefile (gcc; no GPU needed)."""
    import subprocess
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        from_abi = _abi()
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        L.orc_boris_run.restype = C.c_int
        L.orc_boris_run.argtypes = [C.POINTER(from_abi.RunDesc), C.POINTER(from_abi.FieldDesc),
                                    C.POINTER(from_abi.FieldDesc), C.POINTER(FieldCB), C.POINTER(FieldCB),
                                    C.POINTER(TermCB), P, P, P, C.c_int64, C.c_int, C.c_int64, P, P, P, P, P]
        L.orc_gc_run.restype = C.c_int
        L.orc_gc_run.argtypes = [C.POINTER(from_abi.GCDesc), C.POINTER(from_abi.FieldDesc),
                                 C.POINTER(from_abi.FieldDesc), C.POINTER(FieldCB), C.POINTER(FieldCB),
                                 C.POINTER(TermCB), P, P, P, P, P, P, C.c_int64, C.c_int, C.c_int64, P, P, P, P, P]
        L.orc_hybrid_run.restype = C.c_int
        L.orc_hybrid_run.argtypes = [C.POINTER(from_abi.HybridDesc), C.POINTER(from_abi.FieldDesc),
                                     C.POINTER(from_abi.FieldDesc), C.POINTER(FieldCB), C.POINTER(FieldCB),
                                     C.POINTER(TermCB), P, C.c_int64, C.c_int, C.c_int64, C.c_int64, P, P, P, P,
                                     P, P, P, P]
        L.orc_detect.restype = C.c_int
        L.orc_detect.argtypes = [P, P, C.c_int32, P, C.c_int64, P, C.c_int32, P, C.c_double, P, P, P, P]
        L.orc_trig.restype = C.c_int
        L.orc_trig.argtypes = [P, P, C.c_int64, P, P, P]
        L.orc_gc_roundtrip.restype = C.c_int
        L.orc_gc_roundtrip.argtypes = [C.POINTER(from_abi.FieldDesc), C.POINTER(from_abi.FieldDesc), P,
                                       C.c_int64, C.c_double, C.c_double, C.c_double, P]
        L.orc_gc_prepare.restype = C.c_int
        L.orc_gc_prepare.argtypes = [C.POINTER(from_abi.FieldDesc), C.POINTER(from_abi.FieldDesc),
                                     C.POINTER(FieldCB), C.POINTER(FieldCB), P, C.c_int64, C.c_double,
                                     C.c_double, C.c_double, P, P]
        L.orc_gc_to_full.restype = C.c_int
        L.orc_gc_to_full.argtypes = [C.POINTER(from_abi.FieldDesc), C.POINTER(from_abi.FieldDesc),
                                     C.POINTER(FieldCB), C.POINTER(FieldCB), P, P, C.c_int64, C.c_double,
                                     C.c_double, C.c_double, P, C.c_double, P]
        L.orc_field_eval.restype = C.c_int
        L.orc_field_eval.argtypes = [C.POINTER(from_abi.FieldDesc), C.POINTER(FieldCB), P, C.c_int64,
                                     C.c_double, P, P]
        L.orc_boris_counts.restype = C.c_int
        L.orc_boris_counts.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int64, C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_max_threads.restype = C.c_int
        L.orc_boris_jvp.restype = C.c_int
        L.orc_boris_jvp.argtypes = [C.POINTER(from_abi.RunDesc), C.POINTER(from_abi.FieldDesc),
                                    C.POINTER(from_abi.FieldDesc), P, P, P, P, P, C.c_int64, C.c_int, P, P]
        _lib = L
    return _lib


def _abi():
    import importlib.util
    import sys
    mod = sys.modules.get("testparticle_b200._abi")
    if mod is not None:
        return mod
    p = HERE.parent / "testparticle.jl_b200" / "_abi.py"
    spec = importlib.util.spec_from_file_location("_tp_oracle_abi", p)
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def field_callback(fn: Callable, jac: Optional[Callable] = None) -> FieldCB:
    """Wrap fn(x: ndarray(3), t) -> 3-vector (and jac(x, t) -> 3x3) as C callbacks."""

    def f(x, t, out, _u):
        v = fn(np.array([x[0], x[1], x[2]]), t)
        out[0], out[1], out[2] = float(v[0]), float(v[1]), float(v[2])

    cb = FieldCB()
    cb.f = FIELD_CB(f)
    if jac is not None:
        def j(x, t, out, _u):
            J = np.asarray(jac(np.array([x[0], x[1], x[2]]), t), dtype=float).reshape(9)
            for k in range(9):
                out[k] = J[k]
        cb.j = JAC_CB(j)
    else:
        cb.j = JAC_CB()
    cb._keep = (cb.f, cb.j)
    return cb


def term_callback(fn: Callable) -> TermCB:
    """Wrap isoutside(u: ndarray, t) -> bool as a C callback."""

    def f(u, n, t, _u):
        return 1 if fn(np.array([u[k] for k in range(n)]), t) else 0

    cb = TermCB()
    cb.f = OUT_CB(f)
    cb._keep = cb.f
    return cb


@dataclass
class OracleResult:
    nsaved: np.ndarray
    retcode: np.ndarray
    nsteps: np.ndarray
    t: np.ndarray      # packed
    u: np.ndarray      # packed (total, width)

    @property
    def offsets(self):
        o = np.zeros(self.nsaved.size + 1, dtype=np.int64)
        np.cumsum(self.nsaved, out=o[1:])
        return o

    def traj(self, i):
        o = self.offsets
        return self.t[o[i]:o[i + 1]], self.u[o[i]:o[i + 1]]

    def final_states(self):
        o = self.offsets
        return self.u[o[1:] - 1]


def _pack(t_sm, u_sm, nsaved, W, n):
    tot = int(nsaved.sum())
    t = np.empty(tot)
    u = np.empty((tot, W))
    k = 0
    for i in range(n):
        m = int(nsaved[i])
        t[k:k + m] = t_sm[:m, i]
        u[k:k + m] = u_sm[:m, :, i]
        k += m
    return t, u


def _field_arg(f):
    """(descriptor, callback) for a package field object or a Python callable."""
    if f is None:
        return None, None
    if callable(f) and not hasattr(f, "descriptor"):
        return None, field_callback(f)
    if isinstance(f, tuple) and len(f) == 2 and callable(f[0]):
        return None, field_callback(f[0], f[1])
    d = f.descriptor()
    d._keep = f.keepalive()
    return d, None


def boris_run(desc, E, B, u0: np.ndarray, dt_i=None, tend_i=None, nthreads: int = 0,
              isoutside: Optional[Callable] = None, nslots: int = 0) -> OracleResult:
    """Ensemble solve on the CPU; E/B are package fields or Python callables."""
    L = lib()
    u0 = np.ascontiguousarray(u0, dtype=np.float64)
    n = u0.shape[0]
    W = 6 + 6 * bool(desc.save_fields) + 4 * bool(desc.save_work)
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    tcb = term_callback(isoutside) if isoutside is not None else None
    dt_i = None if dt_i is None else np.ascontiguousarray(dt_i, dtype=np.float64)
    tend_i = None if tend_i is None else np.ascontiguousarray(tend_i, dtype=np.float64)
    if nthreads <= 0 and (Ecb is not None or Bcb is not None or tcb is not None):
        nthreads = 1  # Python callbacks hold the GIL
    if nslots <= 0:
        nslots = 16
    for _ in range(3):
        t_sm = np.empty((nslots, n))
        u_sm = np.empty((nslots, W, n))
        nsaved = np.empty(n, dtype=np.int32)
        rc = np.empty(n, dtype=np.int8)
        nst = np.empty(n, dtype=np.int64)
        code = L.orc_boris_run(C.byref(desc), C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None,
                               C.byref(Ecb) if Ecb else None, C.byref(Bcb) if Bcb else None,
                               C.byref(tcb) if tcb else None, _ptr(u0), _ptr(dt_i), _ptr(tend_i), n,
                               int(nthreads), nslots, _ptr(t_sm), _ptr(u_sm), _ptr(nsaved), _ptr(rc),
                               _ptr(nst))
        if code == -6:  # overflow: grow and rerun
            nslots = int(nsaved.max())
            continue
        if code == -1:
            raise ValueError("oracle: ArgumentError")
        if code != 0:
            raise RuntimeError(f"oracle status {code}")
        t, u = _pack(t_sm, u_sm, nsaved, W, n)
        return OracleResult(nsaved, rc, nst, t, u)
    raise RuntimeError("oracle: output sizing failed")


def boris_jvp(desc, E, B, u0: np.ndarray, du0=None, dE_nodes=None, dB_nodes=None, dparam=None,
              nthreads: int = 0):
    """Final save (x_N, v_N) of the fixed-step Boris solve and its directional
    derivative along (du0, node-value tangents of grid fields, parameter
    tangents [E then B: dipole moment, else uniform offset]).  E/B are
    package field objects (analytic kinds or grids).  Returns (uN, duN), N x 6.
    """
    L = lib()
    u0 = np.ascontiguousarray(u0, dtype=np.float64)
    n = u0.shape[0]
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    if Ecb is not None or Bcb is not None:
        raise TypeError("boris_jvp needs package field objects, not callables")

    def arr(a, shape=None):
        if a is None:
            return None
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 4:  # (3, nx, ny, nz) grid tangent: the field's column-major layout
            a = np.asfortranarray(a).ravel(order="F")
        return np.ascontiguousarray(a)

    du0, dEn, dBn, dp = arr(du0), arr(dE_nodes), arr(dB_nodes), arr(dparam)
    uN = np.empty((n, 6))
    duN = np.empty((n, 6))
    code = L.orc_boris_jvp(C.byref(desc), C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None, _ptr(u0),
                           _ptr(du0), _ptr(dEn), _ptr(dBn), _ptr(dp), n, int(nthreads), _ptr(uN), _ptr(duN))
    if code == -1:
        raise ValueError("oracle: ArgumentError")
    if code != 0:
        raise RuntimeError(f"oracle status {code}")
    return uN, duN


def gc_run(desc, E, B, y0: np.ndarray, q_i=None, q2m_i=None, mu_i=None, nthreads: int = 0,
           isoutside: Optional[Callable] = None, nslots: int = 0, dt_i=None, tend_i=None) -> OracleResult:
    L = lib()
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    n = y0.shape[0]
    W = 4 + 6 * bool(desc.save_fields) + 4 * bool(desc.save_work)
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    tcb = term_callback(isoutside) if isoutside is not None else None
    conv = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
            for a in (q_i, q2m_i, mu_i, dt_i, tend_i)]
    if nthreads <= 0 and (Ecb is not None or Bcb is not None or tcb is not None):
        nthreads = 1
    if nslots <= 0:
        nslots = 64
    for _ in range(3):
        t_sm = np.empty((nslots, n))
        u_sm = np.empty((nslots, W, n))
        nsaved = np.empty(n, dtype=np.int32)
        rc = np.empty(n, dtype=np.int8)
        nst = np.empty(n, dtype=np.int64)
        code = L.orc_gc_run(C.byref(desc), C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None,
                            C.byref(Ecb) if Ecb else None, C.byref(Bcb) if Bcb else None,
                            C.byref(tcb) if tcb else None, _ptr(y0), *[_ptr(a) for a in conv], n,
                            int(nthreads), nslots, _ptr(t_sm), _ptr(u_sm), _ptr(nsaved), _ptr(rc), _ptr(nst))
        if code == -6:
            nslots = int(nsaved.max())
            continue
        if code == -1:
            raise ValueError("oracle: ArgumentError")
        if code != 0:
            raise RuntimeError(f"oracle status {code}")
        t, u = _pack(t_sm, u_sm, nsaved, W, n)
        return OracleResult(nsaved, rc, nst, t, u)
    raise RuntimeError("oracle: output sizing failed")


def hybrid_run(desc, E, B, u0: np.ndarray, nthreads: int = 0, isoutside: Optional[Callable] = None):
    """Adaptive hybrid ensemble on the CPU -> (OracleResult, adiabaticity OracleResult or None);
    the adiabaticity rows are (value, mode) with mode 0 = GC, 1 = FO."""
    L = lib()
    u0 = np.ascontiguousarray(u0, dtype=np.float64)
    n = u0.shape[0]
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    tcb = term_callback(isoutside) if isoutside is not None else None
    if nthreads <= 0 and (Ecb is not None or Bcb is not None or tcb is not None):
        nthreads = 1
    want = bool(desc.save_adiabaticity)
    nslots, aslots = 64, 64
    for _ in range(3):
        t_sm = np.empty((nslots, n))
        u_sm = np.empty((nslots, 6, n))
        nsaved = np.zeros(n, dtype=np.int32)
        rc = np.empty(n, dtype=np.int8)
        nst = np.empty(n, dtype=np.int64)
        at = np.empty((aslots, n)) if want else None
        av = np.empty((aslots, 2, n)) if want else None
        na = np.zeros(n, dtype=np.int32) if want else None
        code = L.orc_hybrid_run(C.byref(desc), C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None,
                                C.byref(Ecb) if Ecb else None, C.byref(Bcb) if Bcb else None,
                                C.byref(tcb) if tcb else None, _ptr(u0), n, int(nthreads), nslots, aslots,
                                _ptr(t_sm), _ptr(u_sm), _ptr(nsaved), _ptr(rc), _ptr(nst), _ptr(at), _ptr(av),
                                _ptr(na))
        if code == -6:
            nslots = max(nslots, int(nsaved.max()))
            if want:
                aslots = max(aslots, int(na.max()))
            continue
        if code == -1:
            raise ValueError("oracle: ArgumentError")
        if code != 0:
            raise RuntimeError(f"oracle status {code}")
        t, u = _pack(t_sm, u_sm, nsaved, 6, n)
        res = OracleResult(nsaved, rc, nst, t, u)
        ares = None
        if want:
            ta, ua = _pack(at, av, na, 2, n)
            ares = OracleResult(na, rc, nst, ta, ua)
        return res, ares
    raise RuntimeError("oracle: output sizing failed")


def detect(t, u, nsaved, surfaces, weights=None, weight: float = 1.0):
    """Detector restatement over packed trajectories -> (sums (ns, 4), counts (ns,),
    rows (total, 4), first (n, 6) for surfaces[0]); surfaces are package Surface objects."""
    from_abi = _abi()
    t = np.ascontiguousarray(t, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    ns = np.ascontiguousarray(nsaved, dtype=np.int32)
    n = ns.size
    descs = (from_abi.Surface * len(surfaces))(*[sf.descriptor() for sf in surfaces])
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    sums = np.empty((len(surfaces), 4))
    counts = np.empty(len(surfaces), dtype=np.int64)
    first = np.empty((n, 6))
    L = lib()
    L.orc_detect(_ptr(t), _ptr(u), u.shape[1], _ptr(ns), n, C.cast(descs, C.c_void_p), len(surfaces), _ptr(w),
                 float(weight), _ptr(sums), _ptr(counts), None, _ptr(first))
    rows = np.empty((int(counts.sum()), 4))
    L.orc_detect(_ptr(t), _ptr(u), u.shape[1], _ptr(ns), n, C.cast(descs, C.c_void_p), len(surfaces), _ptr(w),
                 float(weight), None, None, _ptr(rows), None)
    return sums, counts, rows, first


def trig(x: np.ndarray, y: np.ndarray):
    """(sin x, cos x, atan2(y, x)) of the portable trigonometry (hybrid gyrophase, Multistep rotation)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    s, c, a = np.empty_like(x), np.empty_like(x), np.empty_like(x)
    lib().orc_trig(_ptr(x), _ptr(y), x.size, _ptr(s), _ptr(c), _ptr(a))
    return s, c, a


def gc_roundtrip(E, B, xv: np.ndarray, q: float, m: float, t: float = 0.0) -> np.ndarray:
    """Full orbit -> guiding centre -> full orbit, (n, 6) -> (n, 6)."""
    xv = np.ascontiguousarray(np.atleast_2d(xv), dtype=np.float64)
    Ed, _ = _field_arg(E)
    Bd, _ = _field_arg(B)
    out = np.empty_like(xv)
    code = lib().orc_gc_roundtrip(C.byref(Ed), C.byref(Bd), _ptr(xv), xv.shape[0], float(q), float(m), float(t),
                                  _ptr(out))
    if code != 0:
        raise RuntimeError(f"oracle status {code}")
    return out


def gc_prepare(E, B, xv: np.ndarray, q: float, m: float, t: float = 0.0):
    L = lib()
    xv = np.ascontiguousarray(np.atleast_2d(xv), dtype=np.float64)
    n = xv.shape[0]
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    y0 = np.empty((n, 4))
    mu = np.empty(n)
    code = L.orc_gc_prepare(C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None,
                            C.byref(Ecb) if Ecb else None, C.byref(Bcb) if Bcb else None, _ptr(xv), n,
                            float(q), float(m), float(t), _ptr(y0), _ptr(mu))
    if code != 0:
        raise RuntimeError(f"oracle status {code}")
    return y0, mu


def gc_to_full(E, B, y: np.ndarray, mu, q: float, m: float, phase=0.0, t: float = 0.0):
    """gc_to_full restatement at rows of y (N, 4) -> (N, 6); phase scalar or (N,)."""
    L = lib()
    y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
    n = y.shape[0]
    mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, dtype=np.float64), (n,)))
    ph = np.asarray(phase, dtype=np.float64)
    ph_i = np.ascontiguousarray(np.broadcast_to(ph, (n,))) if ph.ndim else None
    Ed, Ecb = _field_arg(E)
    Bd, Bcb = _field_arg(B)
    out = np.empty((n, 6))
    code = L.orc_gc_to_full(C.byref(Ed) if Ed else None, C.byref(Bd) if Bd else None,
                            C.byref(Ecb) if Ecb else None, C.byref(Bcb) if Bcb else None, _ptr(y), _ptr(mu), n,
                            float(q), float(m), float(ph) if ph_i is None else 0.0, _ptr(ph_i), float(t),
                            _ptr(out))
    if code != 0:
        raise RuntimeError(f"oracle status {code}")
    return out


def field_eval(F, x: np.ndarray, t: float = 0.0, jacobian: bool = False):
    L = lib()
    x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
    n = x.shape[0]
    d, cb = _field_arg(F)
    out = np.empty((n, 3))
    J = np.empty((n, 3, 3)) if jacobian else None
    code = L.orc_field_eval(C.byref(d) if d else None, C.byref(cb) if cb else None, _ptr(x), n, float(t),
                            _ptr(out), _ptr(J))
    if code != 0:
        raise RuntimeError(f"oracle status {code}")
    return (out, J) if jacobian else out


def boris_counts(t0, t1, dt, maxiters, ssi, save_start=True, save_end=True, save_everystep=True):
    L = lib()
    nt = C.c_int64()
    nout = C.c_int64()
    code = L.orc_boris_counts(t0, t1, dt, maxiters, ssi, int(save_start), int(save_end), int(save_everystep),
                              C.byref(nt), C.byref(nout))
    if code != 0:
        raise ValueError("ArgumentError")
    return nt.value, nout.value


def max_threads() -> int:
    return int(lib().orc_max_threads())
