"""Thin Python side of the C ABI: contexts, device fields, host-buffer runs.

Everything computational happens in libtpb200.so; this module only marshals
numpy buffers and descriptors and turns status codes into the reference's
exception types (TP_E_ARG -> ValueError, the Python spelling of Julia's
ArgumentError; the others -> RuntimeError).
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from dataclasses import dataclass

import numpy as np

from . import _abi


class ArgumentError(ValueError):
    """The reference's ArgumentError (invalid dt, nt > maxiters, bad order...)."""


class DeviceError(RuntimeError):
    """A CUDA, timeout or capacity failure reported by the library."""


def _check(lib, ctx, code: int, what: str):
    if code == _abi.TP_OK:
        return
    msg = lib.tp_last_error(ctx).decode() if ctx else ""
    text = f"{what}: {msg} (status {code})"
    if code == _abi.TP_E_ARG:
        raise ArgumentError(text)
    if code == _abi.TP_E_UNSUPPORTED:
        raise NotImplementedError(text)
    raise DeviceError(text)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One library context (device, stream) per device, shared by the process."""

    _lock = threading.Lock()
    _by_device: dict[int, "Context"] = {}

    def __init__(self, device: int):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        code = self.lib.tp_ctx_create(int(device), C.byref(h))
        if code != _abi.TP_OK:
            raise DeviceError(f"tp_ctx_create(device={device}) failed with status {code}")
        self.handle = h
        self.device = device
        self._fields: dict[int, tuple] = {}
        weakref.finalize(self, self.lib.tp_ctx_destroy, h)

    @classmethod
    def get(cls, device: int = 0) -> "Context":
        with cls._lock:
            ctx = cls._by_device.get(device)
            if ctx is None:
                ctx = cls(device)
                cls._by_device[device] = ctx
            return ctx

    # ------------------------------------------------------------ fields
    def field(self, f) -> C.c_void_p:
        """Device handle of a field object (uploaded once, cached by identity)."""
        key = id(f)
        hit = self._fields.get(key)
        if hit is not None and hit[0]() is f:
            return hit[1]
        desc = f.descriptor()
        keep = f.keepalive()  # noqa: F841 - keeps grid data alive through the upload
        h = C.c_void_p()
        _check(self.lib, self.handle, self.lib.tp_field_create(self.handle, C.byref(desc), C.byref(h)),
               "tp_field_create")
        lib = self.lib

        def _drop(k=key, handle=h, fields=self._fields):
            fields.pop(k, None)
            lib.tp_field_destroy(handle)

        try:
            ref = weakref.ref(f, lambda _r: _drop())
        except TypeError:  # objects without weakref support: keep for the context lifetime
            ref = (lambda obj=f: obj)
        self._fields[key] = (ref, h)
        return h

    # ------------------------------------------------------------ runs
    def boris_run(self, desc: _abi.RunDesc, E, B, u0: np.ndarray, dt_i=None, tend_i=None):
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        n = u0.shape[0]
        assert u0.shape == (n, 6)
        dt_i = None if dt_i is None else np.ascontiguousarray(dt_i, dtype=np.float64)
        tend_i = None if tend_i is None else np.ascontiguousarray(tend_i, dtype=np.float64)
        res = C.c_void_p()
        code = self.lib.tp_boris_run(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0),
                                     _ptr(dt_i), _ptr(tend_i), n, C.byref(res))
        _check(self.lib, self.handle, code, "tp_boris_run")
        return self._collect(res)

    def gc_run(self, desc: _abi.GCDesc, E, B, y0: np.ndarray, q_i=None, q2m_i=None, mu_i=None,
               dt_i=None, tend_i=None):
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        n = y0.shape[0]
        assert y0.shape == (n, 4)
        conv = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (q_i, q2m_i, mu_i, dt_i, tend_i)]
        res = C.c_void_p()
        code = self.lib.tp_gc_run(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(y0),
                                  *[_ptr(a) for a in conv], n, C.byref(res))
        _check(self.lib, self.handle, code, "tp_gc_run")
        return self._collect(res)

    def slots(self, desc: _abi.RunDesc, n: int, dt_i=None, tend_i=None) -> int:
        """Save slots per trajectory a full-orbit run needs (-1: unknown, adaptive without cap)."""
        dt_i = None if dt_i is None else np.ascontiguousarray(dt_i, dtype=np.float64)
        tend_i = None if tend_i is None else np.ascontiguousarray(tend_i, dtype=np.float64)
        ns = C.c_int64()
        _check(self.lib, self.handle, self.lib.tp_boris_slots(C.byref(desc), _ptr(dt_i), _ptr(tend_i), n,
                                                              C.byref(ns)), "tp_boris_slots")
        return ns.value

    def boris_run_device(self, desc: _abi.RunDesc, E, B, u0, dt_i, tend_i, n: int, nslots: int, t_out,
                         u_out, nsaved, retcode, nsteps, status, stream: int = 0):
        """Device-buffer run: every array argument is a device pointer (int) or None."""
        code = self.lib.tp_boris_run_device(self.handle, C.byref(desc), self.field(E), self.field(B), u0,
                                            dt_i, tend_i, int(n), int(nslots), t_out, u_out, nsaved, retcode,
                                            nsteps, status, stream)
        _check(self.lib, self.handle, code, "tp_boris_run_device")

    def gc_prepare(self, E, B, xv: np.ndarray, q: float, m: float, t: float = 0.0):
        xv = np.ascontiguousarray(xv, dtype=np.float64)
        n = xv.shape[0]
        y0 = np.empty((n, 4))
        mu = np.empty(n)
        code = self.lib.tp_gc_prepare(self.handle, self.field(E), self.field(B), _ptr(xv), n, float(q),
                                      float(m), float(t), _ptr(y0), _ptr(mu))
        _check(self.lib, self.handle, code, "tp_gc_prepare")
        return y0, mu

    def _collect(self, res: C.c_void_p) -> "RunResult":
        lib = self.lib
        try:
            n = C.c_int64()
            w = C.c_int32()
            tot = C.c_int64()
            lib.tp_result_info(res, C.byref(n), C.byref(w), C.byref(tot))
            nsaved = np.empty(n.value, dtype=np.int32)
            retcode = np.empty(n.value, dtype=np.int8)
            nsteps = np.empty(n.value, dtype=np.int64)
            t = np.empty(tot.value, dtype=np.float64)
            u = np.empty((tot.value, w.value), dtype=np.float64)
            lib.tp_result_copy(res, _ptr(nsaved), _ptr(retcode), _ptr(nsteps), _ptr(t), _ptr(u))
            ms = C.c_double()
            lib.tp_result_elapsed_ms(res, C.byref(ms))
        finally:
            lib.tp_result_destroy(res)
        return RunResult(nsaved, retcode, nsteps, t, u, ms.value)


@dataclass
class RunResult:
    nsaved: np.ndarray
    retcode: np.ndarray
    nsteps: np.ndarray
    t: np.ndarray        # packed save times
    u: np.ndarray        # packed states (total, width)
    elapsed_ms: float    # device time of the kernels

    @property
    def offsets(self) -> np.ndarray:
        o = np.zeros(self.nsaved.size + 1, dtype=np.int64)
        np.cumsum(self.nsaved, out=o[1:])
        return o
