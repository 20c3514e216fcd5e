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
        self._closed = [False]
        self.tuned_keys: set = set()
        # at exit the context is released before module teardown frees the
        # field objects: release their device copies first, and make the
        # field callbacks that run later do nothing
        weakref.finalize(self, Context._close, self.lib, h, self._fields, self._closed)

    @staticmethod
    def _close(lib, handle, fields, closed):
        closed[0] = True
        for _ref, fh in list(fields.values()):
            lib.tp_field_destroy(fh)
        fields.clear()
        lib.tp_ctx_destroy(handle)

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

        def _drop(k=key, handle=h, fields=self._fields, closed=self._closed):
            if closed[0] or fields.pop(k, None) is None:
                return
            lib.tp_field_destroy(handle)

        try:
            ref = weakref.ref(f, lambda _r: _drop())
        except TypeError:  # objects without weakref support: keep for the context lifetime
            ref = (lambda obj=f: obj)
        self._fields[key] = (ref, h)
        return h

    # ------------------------------------------------------------ runs
    def boris_run(self, desc: _abi.RunDesc, E, B, u0: np.ndarray, dt_i=None, tend_i=None, pipelined=True):
        """Full-orbit solve of host arrays.  With a known save count it runs
        through tp_boris_run_host (chunks, results copied while later chunks
        compute); otherwise, or with pipelined=False, through tp_boris_run and
        tp_result_copy.  Both give the same results bit for bit."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        n = u0.shape[0]
        assert u0.shape == (n, 6)
        dt_i = None if dt_i is None else np.ascontiguousarray(dt_i, dtype=np.float64)
        tend_i = None if tend_i is None else np.ascontiguousarray(tend_i, dtype=np.float64)
        res = C.c_void_p()
        width = 6 + 6 * bool(desc.save_fields) + 4 * bool(desc.save_work)
        ns = C.c_int64(-1)
        # slots per trajectory (an invalid descriptor is reported by the run itself)
        if n > 0 and self.lib.tp_boris_slots(C.byref(desc), _ptr(dt_i), _ptr(tend_i), n, C.byref(ns)) != _abi.TP_OK:
            ns.value = -1
        if pipelined and ns.value >= 0 and n > 0:
            return self.boris_run_host(desc, E, B, u0, dt_i, tend_i, n * ns.value)
        code = self.lib.tp_boris_run(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0),
                                     _ptr(dt_i), _ptr(tend_i), n, C.byref(res))
        _check(self.lib, self.handle, code, "tp_boris_run")
        return self._collect(res)

    def boris_run_host(self, desc: _abi.RunDesc, E, B, u0: np.ndarray, dt_i, tend_i, cap_rows: int):
        """tp_boris_run_host: one kernel, with each finished chunk of particles
        copied and packed into the returned arrays while the kernel runs.  The
        row arrays are allocated at cap_rows and not touched beforehand: the
        library's packing threads fault their pages in while the GPU is busy."""
        n = u0.shape[0]
        width = 6 + 6 * bool(desc.save_fields) + 4 * bool(desc.save_work)
        nsaved = np.empty(n, dtype=np.int32)
        retcode = np.empty(n, dtype=np.int8)
        nsteps = np.empty(n, dtype=np.int64)
        t = np.empty(max(cap_rows, 1), dtype=np.float64)
        u = np.empty((max(cap_rows, 1), width), dtype=np.float64)
        tot = C.c_int64()
        ms = C.c_double()
        code = self.lib.tp_boris_run_host(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0),
                                          _ptr(dt_i), _ptr(tend_i), n, cap_rows, _ptr(nsaved), _ptr(retcode),
                                          _ptr(nsteps), _ptr(t), _ptr(u), C.byref(tot), C.byref(ms))
        _check(self.lib, self.handle, code, "tp_boris_run_host")
        return RunResult(nsaved, retcode, nsteps, t[:tot.value], u[:tot.value], ms.value)

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

    def hybrid_run(self, desc: _abi.HybridDesc, E, B, u0: np.ndarray, adiabaticity: bool = True):
        """tp_hybrid_run -> (RunResult, RunResult of (value, mode) checks or None)."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        n = u0.shape[0]
        assert u0.shape == (n, 6)
        res, ares = C.c_void_p(), C.c_void_p()
        code = self.lib.tp_hybrid_run(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0), n,
                                      C.byref(res), C.byref(ares) if adiabaticity else None)
        _check(self.lib, self.handle, code, "tp_hybrid_run")
        main = self._collect(res)
        return main, (self._collect(ares) if adiabaticity and ares.value else None)

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

    def field_update(self, f, data) -> None:
        """Replace the node values of a grid field already on the device (tp_field_update).

        `data` is a (3, nx, ny, nz) array in the field's dtype, or an int
        device pointer to the same layout (component fastest).
        """
        h = self.field(f)
        if isinstance(data, int):
            ptr = C.c_void_p(data)
        else:
            a = np.asfortranarray(np.asarray(data, dtype=f.data.dtype))
            if a.shape != f.data.shape:
                raise ValueError("field_update: shape differs from the field's grid")
            f.data = a
            ptr = a.ctypes.data_as(C.c_void_p)
        _check(self.lib, self.handle, self.lib.tp_field_update(h, ptr), "tp_field_update")

    # ------------------------------------------------------------ tuning, graphs
    def autotune(self, desc: _abi.RunDesc, E, B, u0: np.ndarray, max_steps: int = 200) -> dict:
        """Time the candidate launch shapes on a sample of the run (tp_autotune); later runs of the
        same kernel variant with block = 0 / schedule = "auto" use the fastest."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        r = _abi.TuneResult()
        code = self.lib.tp_autotune(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0),
                                    u0.shape[0], int(max_steps), C.byref(r))
        _check(self.lib, self.handle, code, "tp_autotune")
        return {"block": r.block, "schedule": {1: "static", 2: "queue"}.get(r.schedule, "auto"),
                "particles_per_thread": r.particles_per_thread, "ms": r.ms, "ms_default": r.ms_default,
                "candidates": r.candidates}

    def boris_graph(self, desc: _abi.RunDesc, E, B, u0, dt_i, tend_i, n: int, nslots: int, t_out, u_out, nsaved,
                    retcode, nsteps, status) -> "Graph":
        """A solve over fixed device buffers (pointers, as boris_run_device) captured as a CUDA graph."""
        h = C.c_void_p()
        code = self.lib.tp_boris_graph_create(self.handle, C.byref(desc), self.field(E), self.field(B), u0, dt_i,
                                              tend_i, int(n), int(nslots), t_out, u_out, nsaved, retcode, nsteps,
                                              status, C.byref(h))
        _check(self.lib, self.handle, code, "tp_boris_graph_create")
        return Graph(self, h, E, B)

    # ------------------------------------------------------------ adjoint
    def adjoint_forward(self, desc: _abi.AdjDesc, E, B, u0: np.ndarray):
        """Final save (x_N, v_N) (N x 6) of a fixed-step Boris solve and the tape of its adjoint."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        n = u0.shape[0]
        assert u0.shape == (n, 6)
        uf = np.empty((n, 6))
        h = C.c_void_p()
        code = self.lib.tp_adjoint_forward(self.handle, C.byref(desc), self.field(E), self.field(B), _ptr(u0), n,
                                           _ptr(uf), C.byref(h))
        _check(self.lib, self.handle, code, "tp_adjoint_forward")
        return uf, Tape(self, h, n, E, B)

    def adjoint_forward_device(self, desc: _abi.AdjDesc, E, B, u0: int, n: int, u_final: int,
                               stream: int = 0) -> "Tape":
        """Device-buffer forward: u0 and u_final are device pointers (N x 6 float64)."""
        h = C.c_void_p()
        code = self.lib.tp_adjoint_forward_device(self.handle, C.byref(desc), self.field(E), self.field(B), u0,
                                                  int(n), u_final, C.byref(h), stream)
        _check(self.lib, self.handle, code, "tp_adjoint_forward_device")
        return Tape(self, h, n, E, B)

    def gc_prepare(self, E, B, xv: np.ndarray, q: float, m: float, t: float = 0.0):
        xv = np.ascontiguousarray(xv, dtype=np.float64)
        n = xv.shape[0]
        y0 = np.empty((n, 4))
        mu = np.empty(n)
        code = self.lib.tp_gc_prepare(self.handle, self.field(E), self.field(B), _ptr(xv), n, float(q),
                                      float(m), float(t), _ptr(y0), _ptr(mu))
        _check(self.lib, self.handle, code, "tp_gc_prepare")
        return y0, mu

    def gc_to_full(self, E, B, y: np.ndarray, mu, q: float, m: float, phase=0.0, t: float = 0.0) -> np.ndarray:
        """tp_gc_to_full: full-orbit states (N, 6) of guiding-centre rows y (N, 4)."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.shape[0]
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, dtype=np.float64), (n,)))
        ph = np.asarray(phase, dtype=np.float64)
        ph_i = np.ascontiguousarray(np.broadcast_to(ph, (n,))) if ph.ndim else None
        xv = np.empty((n, 6))
        code = self.lib.tp_gc_to_full(self.handle, self.field(E), self.field(B), _ptr(y), _ptr(mu), n, float(q),
                                      float(m), float(ph) if ph_i is None else 0.0, _ptr(ph_i), float(t), _ptr(xv))
        _check(self.lib, self.handle, code, "tp_gc_to_full")
        return xv

    def eval_points(self, E, B, u: np.ndarray, t: np.ndarray, *, gc: bool, want: int, q2m=0.0, m=0.0, q=0.0,
                    mu=0.0) -> np.ndarray:
        """tp_eval_points: E, B (want & 1) and work rates (want & 2) at n states.  q2m, m, q and mu are
        scalars or arrays of one value per state (tp_eval_points_params: still one launch)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64).reshape(-1)
        if u.ndim != 2 or u.shape[0] != t.size:
            raise ValueError("u must be (n, width) with one time per state")
        d = _abi.PointsDesc()
        d.kind = _abi.TP_POINTS_GC if gc else _abi.TP_POINTS_FULL_ORBIT
        d.want = int(want)
        d.stride = int(u.shape[1])
        per = {}
        for name, val in (("q2m", q2m), ("m", m), ("q", q), ("mu", mu)):
            if np.ndim(val) == 0:
                setattr(d, name, float(val))
            else:
                a = np.ascontiguousarray(val, dtype=np.float64).reshape(-1)
                if a.size != t.size:
                    raise ValueError(f"{name} must be a scalar or one value per state")
                per[name] = a
        wout = 6 * (want & 1) + 4 * ((want >> 1) & 1)
        out = np.empty((t.size, wout))
        if per:
            code = self.lib.tp_eval_points_params(self.handle, C.byref(d), self.field(E), self.field(B), _ptr(u),
                                                  _ptr(t), _ptr(per.get("q2m")), _ptr(per.get("m")),
                                                  _ptr(per.get("q")), _ptr(per.get("mu")), t.size, _ptr(out))
        else:
            code = self.lib.tp_eval_points(self.handle, C.byref(d), self.field(E), self.field(B), _ptr(u),
                                           _ptr(t), t.size, _ptr(out))
        _check(self.lib, self.handle, code, "tp_eval_points")
        return out

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


def _grid_nodes(f) -> int:
    d = getattr(f, "data", None)
    return int(np.prod(d.shape[1:])) if d is not None and getattr(d, "ndim", 0) == 4 else 0


@dataclass
class AdjointGrads:
    u0: np.ndarray                 # dL/du0, N x 6
    E: object                      # dL/d(E node values), (3, nx, ny, nz) float64, or None
    B: object
    param: np.ndarray              # 6: (E, B) dipole moment or uniform-offset gradients


class Tape:
    """Checkpoints of one adjoint forward pass (tp_tape); backward() may run more than once."""

    def __init__(self, ctx: Context, handle: C.c_void_p, n: int, E, B):
        self.ctx, self.handle, self.n = ctx, handle, int(n)
        self.E, self.B = E, B  # the fields must outlive the tape
        self._fin = weakref.finalize(self, ctx.lib.tp_tape_destroy, handle)

    def backward(self, grad_final: np.ndarray, fields: bool = True) -> AdjointGrads:
        lib = self.ctx.lib
        g = np.ascontiguousarray(grad_final, dtype=np.float64)
        assert g.shape == (self.n, 6)
        gu = np.empty((self.n, 6))
        gp = np.empty(6)
        out = []
        for f in (self.E, self.B):
            nodes = _grid_nodes(f) if fields else 0
            out.append(np.empty(3 * nodes, dtype=np.float64) if nodes else None)
        code = lib.tp_adjoint_backward(self.handle, _ptr(g), _ptr(gu), _ptr(out[0]), _ptr(out[1]), _ptr(gp))
        _check(lib, self.ctx.handle, code, "tp_adjoint_backward")
        shaped = [None if a is None else a.reshape(f.data.shape, order="F") for a, f in zip(out, (self.E, self.B))]
        return AdjointGrads(gu, shaped[0], shaped[1], gp)

    def backward_device(self, grad_final: int, grad_u0: int, grad_E=None, grad_B=None, grad_param=None,
                        stream: int = 0) -> None:
        """Device-buffer backward: every argument is a device pointer (int) or None."""
        code = self.ctx.lib.tp_adjoint_backward_device(self.handle, grad_final, grad_u0, grad_E, grad_B,
                                                       grad_param, stream)
        _check(self.ctx.lib, self.ctx.handle, code, "tp_adjoint_backward_device")

    def rerun_device(self, u0: int, u_final: int, stream: int = 0) -> None:
        """Re-record the tape for new initial states (device pointers), reusing its memory."""
        code = self.ctx.lib.tp_tape_rerun_device(self.handle, u0, u_final, stream)
        _check(self.ctx.lib, self.ctx.handle, code, "tp_tape_rerun_device")

    def info(self) -> tuple[int, int]:
        """(device bytes held, steps N)."""
        b, s = C.c_int64(), C.c_int64()
        self.ctx.lib.tp_tape_info(self.handle, C.byref(b), C.byref(s))
        return b.value, s.value

    def segments(self) -> tuple[int, int]:
        """(steps per checkpoint segment, segments): the automatic choice resolved."""
        k, s = C.c_int64(), C.c_int64()
        self.ctx.lib.tp_tape_segments(self.handle, C.byref(k), C.byref(s))
        return k.value, s.value

    def close(self) -> None:
        self._fin()


class Graph:
    """A captured solve (tp_graph); launch(stream) replays it."""

    def __init__(self, ctx: Context, handle: C.c_void_p, E, B):
        self.ctx, self.handle = ctx, handle
        self.E, self.B = E, B  # the fields must outlive the graph
        self._fin = weakref.finalize(self, ctx.lib.tp_graph_destroy, handle)

    def launch(self, stream: int = 0) -> None:
        _check(self.ctx.lib, self.ctx.handle, self.ctx.lib.tp_graph_launch(self.handle, stream), "tp_graph_launch")

    def close(self) -> None:
        self._fin()
