"""torch.autograd.Function over the discrete adjoint of the Boris map.

`boris_final_state(u0, E, B, q2m=..., dt=..., tspan=...)` returns the final
save (x_N, v_N) of solve(TraceProblem(u0, tspan, param), Boris(); dt) for N
particles as an (N, 6) float64 CUDA tensor, differentiable with respect to
u0 and to the tensors inside E and B:

  GridTensor(data, origin, spacing, bc)  node values (3, nx, ny, nz)
  UniformTensor(value)                   a uniform field, value (3,)
  DipoleTensor(moment, center)           a point dipole, moment (3,)

Plain package fields (ZeroField, UniformField, DipoleField,
FieldInterpolator, ...) are accepted as constants.  The forward pass runs
tp_adjoint_forward_device (FP32C push, checkpoints every `checkpoint_every`
steps) on torch's current stream; backward runs tp_adjoint_backward_device.
Node gradients are accumulated in float32 with a power-of-two scale per pass,
returned in float64 by the library, and cast to the data's dtype.

The Julia counterpart is the ChainRulesCore rrule of TestParticleB200.jl.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _abi
from .fields import AbstractField, WrapExtrap, _bc_code
from .runtime import Context


class GridTensor(AbstractField):
    """Trilinear grid field whose node values are a CUDA tensor (3, nx, ny, nz)."""

    def __init__(self, data: torch.Tensor, origin, spacing, bc=None):
        if data.dim() != 4 or data.shape[0] != 3:
            raise ValueError("GridTensor data must be (3, nx, ny, nz)")
        self.data = data
        self.origin = tuple(float(v) for v in origin)
        self.spacing = tuple(float(v) for v in spacing)
        self.bc = bc if bc is not None else WrapExtrap()

    def _device_copy(self, values: torch.Tensor) -> "_GridProxy":
        # (3, nx, ny, nz) column-major == (nz, ny, nx, 3) row-major
        return _GridProxy(self, values.detach().permute(3, 2, 1, 0).contiguous())


class UniformTensor(AbstractField):
    def __init__(self, value: torch.Tensor):
        self.data = value


class DipoleTensor(AbstractField):
    def __init__(self, moment: torch.Tensor, center=(0.0, 0.0, 0.0)):
        from .constants import MU0_OVER_4PI
        self.data = moment
        self.center = tuple(float(c) for c in center)
        self.coef = MU0_OVER_4PI


class _GridProxy(AbstractField):
    """Descriptor of a GridTensor's device values for tp_field_create."""

    def __init__(self, g: GridTensor, dev: torch.Tensor):
        self.g, self.dev = g, dev
        self.n = tuple(int(x) for x in g.data.shape[1:])

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = _abi.TP_FIELD_GRID
        d.bc = _bc_code(self.g.bc)
        d.dtype = _abi.TP_DTYPE_F32 if self.dev.dtype == torch.float32 else _abi.TP_DTYPE_F64
        for k in range(3):
            d.n[k] = self.n[k]
            d.origin[k] = self.g.origin[k]
            d.spacing[k] = self.g.spacing[k]
        d.data = self.dev.data_ptr()
        return d

    def keepalive(self):
        return self.dev


class _ValueProxy(AbstractField):
    def __init__(self, kind: int, value, center=(0.0, 0.0, 0.0), coef=0.0):
        self.kind, self.value, self.center, self.coef = kind, [float(v) for v in value], center, coef

    def descriptor(self):
        d = _abi.FieldDesc()
        d.kind = self.kind
        if self.kind == _abi.TP_FIELD_DIPOLE:
            for k in range(3):
                d.moment[k] = self.value[k]
                d.center[k] = self.center[k]
            d.coef = self.coef
        else:
            for k in range(3):
                d.value[k] = self.value[k]
        return d

    def keepalive(self):
        return None


def _tensor_of(f):
    return f.data if isinstance(f, (GridTensor, UniformTensor, DipoleTensor)) else None


def _proxy(f, values):
    if isinstance(f, GridTensor):
        return f._device_copy(values)
    if isinstance(f, UniformTensor):
        return _ValueProxy(_abi.TP_FIELD_UNIFORM, values.detach().cpu().numpy())
    if isinstance(f, DipoleTensor):
        return _ValueProxy(_abi.TP_FIELD_DIPOLE, values.detach().cpu().numpy(), f.center, f.coef)
    return f


def _run_desc(q2m: float, m: float, dt: float, tspan, checkpoint_every: int, block: int) -> _abi.AdjDesc:
    d = _abi.AdjDesc()
    r = d.run
    r.alg = _abi.TP_ALG_BORIS
    r.order, r.nsub = 2, 1
    r.precision = _abi.TP_PREC_FP32C
    r.t0, r.t1, r.dt = float(tspan[0]), float(tspan[1]), float(dt)
    r.q2m, r.m = float(q2m), float(m)
    r.savestepinterval = 1
    nt = int(np.rint(abs((r.t1 - r.t0) / r.dt))) if r.dt != 0 else 0
    r.maxiters = max(1_000_000, nt)
    r.save_start, r.save_end, r.save_everystep = 0, 1, 0
    r.block = int(block)
    d.checkpoint_every = int(checkpoint_every)
    return d


class BorisAdjointFunction(torch.autograd.Function):
    """(u0, E tensor, B tensor) -> (x_N, v_N); see boris_final_state."""

    @staticmethod
    def forward(ctx, u0, e_val, b_val, spec):
        E_in, B_in, desc, device = spec
        E = _proxy(E_in, e_val)
        B = _proxy(B_in, b_val)
        # the proxies' device copies are made on torch's stream and the field
        # uploads read them on the library's stream
        torch.cuda.current_stream(device).synchronize()
        lib_ctx = Context.get(device)
        u0c = u0.detach().to(torch.float64).contiguous()
        n = u0c.shape[0]
        uf = torch.empty_like(u0c)
        stream = torch.cuda.current_stream(device).cuda_stream
        tape = lib_ctx.adjoint_forward_device(desc, E, B, u0c.data_ptr(), n, uf.data_ptr(), stream)
        ctx.tape, ctx.E_in, ctx.B_in, ctx.E, ctx.B, ctx.device = tape, E_in, B_in, E, B, device
        ctx.u_dtype = u0.dtype
        ctx.e_meta = None if e_val is None else (e_val.shape, e_val.dtype)
        ctx.b_meta = None if b_val is None else (b_val.shape, b_val.dtype)
        return uf

    @staticmethod
    def backward(ctx, g):
        dev = torch.device("cuda", ctx.device)
        g = g.to(torch.float64).contiguous()
        gu = torch.empty_like(g)
        gp = torch.zeros(6, dtype=torch.float64, device=dev)

        def node_buf(f):
            if isinstance(f, GridTensor):
                return torch.empty(3 * int(np.prod(f.data.shape[1:])), dtype=torch.float64, device=dev)
            return None

        gE = node_buf(ctx.E_in) if ctx.needs_input_grad[1] else None
        gB = node_buf(ctx.B_in) if ctx.needs_input_grad[2] else None
        stream = torch.cuda.current_stream(ctx.device).cuda_stream
        ctx.tape.backward_device(g.data_ptr(), gu.data_ptr(), None if gE is None else gE.data_ptr(),
                                 None if gB is None else gB.data_ptr(), gp.data_ptr(), stream)

        def field_grad(f, buf, meta, k):
            if meta is None:
                return None
            shape, dtype = meta
            if isinstance(f, GridTensor):
                if buf is None:
                    return None
                nx, ny, nz = shape[1], shape[2], shape[3]
                return buf.view(nz, ny, nx, 3).permute(3, 2, 1, 0).to(dtype)
            return gp[3 * k:3 * k + 3].to(dtype)

        return (gu.to(ctx.u_dtype), field_grad(ctx.E_in, gE, ctx.e_meta, 0),
                field_grad(ctx.B_in, gB, ctx.b_meta, 1), None)


def boris_final_state(u0: torch.Tensor, E, B, *, q2m: float, dt: float, tspan, m: float = 1.0,
                      checkpoint_every: int = 0, block: int = 0) -> torch.Tensor:
    """Differentiable final save (x_N, v_N), (N, 6) float64, of the fixed-step Boris solve.

    The forward is the FP32C push of EnsembleB200(precision="fp32c") without
    intermediate saves; gradients flow to u0 and to the tensors of GridTensor,
    UniformTensor and DipoleTensor fields.
    """
    if not u0.is_cuda:
        raise ValueError("boris_final_state needs CUDA tensors (the B200 library has no CPU path)")
    device = u0.device.index if u0.device.index is not None else torch.cuda.current_device()
    desc = _run_desc(q2m, m, dt, tspan, checkpoint_every, block)
    return BorisAdjointFunction.apply(u0, _tensor_of(E), _tensor_of(B), (E, B, desc, device))
