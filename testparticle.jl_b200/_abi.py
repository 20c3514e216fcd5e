"""ctypes view of include/tp_abi.h and the loader of libtpb200.so.

The structures mirror the C declarations field for field.  The library is
loaded from this directory; a missing library raises ImportError -- there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libtpb200.so"

TP_ABI_VERSION = 3

TP_OK = 0
TP_E_ARG = -1
TP_E_CUDA = -2
TP_E_TIMEOUT = -3
TP_E_NOMEM = -4
TP_E_UNSUPPORTED = -5
TP_E_OVERFLOW = -6

TP_RET_DEFAULT = 0
TP_RET_SUCCESS = 1
TP_RET_TERMINATED = 2
TP_RET_MAXITERS = 3

TP_FIELD_ZERO = 0
TP_FIELD_UNIFORM = 1
TP_FIELD_AFFINE = 2
TP_FIELD_DIPOLE = 3
TP_FIELD_GRID = 4
TP_FIELD_QUADRATIC = 5
TP_FIELD_SERIES = 6

TP_BC_FILL_NAN = 0
TP_BC_CLAMP = 1
TP_BC_PERIODIC = 2
TP_BC_PERIODIC_INCLUSIVE = 3

TP_ORDER_LINEAR = 0
TP_ORDER_CONSTANT = 1
TP_ORDER_CUBIC = 2

TP_GRID_CARTESIAN = 0
TP_GRID_SPHERICAL = 1
TP_GRID_SPHERICAL_SCALAR = 2

TP_ADIA_CURVATURE = 0
TP_ADIA_GRADB = 1
TP_ADIA_BOTH = 2
TP_ADIA_JACOBIAN = 3

TP_SURF_PLANE = 0
TP_SURF_DISK = 1
TP_SURF_SPHERE = 2

TP_POINTS_FULL_ORBIT = 0
TP_POINTS_GC = 1

TP_DTYPE_F32 = 0
TP_DTYPE_F64 = 1

TP_TERM_SHELL = 1
TP_TERM_BOX = 2
TP_TERM_NAN = 4
TP_TERM_TIME = 8

TP_ALG_BORIS = 0
TP_ALG_MULTISTEP = 1
TP_ALG_ADAPTIVE = 2
TP_ALG_ADAPTIVE_MULTISTEP = 3

TP_PREC_FP64 = 0
TP_PREC_FP32C = 1

TP_SCHED_AUTO = 0
TP_SCHED_STATIC = 1
TP_SCHED_QUEUE = 2

TP_GC_RK4 = 0
TP_GC_RK45 = 1
TP_GC_PREC_FP64 = 0
TP_GC_PREC_FP32RHS = 1

_D3 = C.c_double * 3
_D9 = C.c_double * 9
_I3 = C.c_int64 * 3


class FieldDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("bc", C.c_int32),
        ("dtype", C.c_int32),
        ("reserved", C.c_int32),
        ("value", _D3),
        ("jac", _D9),
        ("rate", _D3),
        ("moment", _D3),
        ("center", _D3),
        ("coef", C.c_double),
        ("n", _I3),
        ("origin", _D3),
        ("spacing", _D3),
        ("data", C.c_void_p),
        ("order", C.c_int32),
        ("geometry", C.c_int32),
        ("ndim", C.c_int32),
        ("dir", C.c_int32),
        ("axis", C.c_void_p * 3),
        ("quad", C.c_double * 27),
        ("nseries", C.c_int64),
        ("series_times", C.c_void_p),
        ("series", C.c_void_p),
    ]


class TermDesc(C.Structure):
    _fields_ = [
        ("flags", C.c_int32),
        ("reserved", C.c_int32),
        ("rmin", C.c_double),
        ("rmax", C.c_double),
        ("lo", _D3),
        ("hi", _D3),
        ("tmax", C.c_double),
    ]


class RunDesc(C.Structure):
    _fields_ = [
        ("alg", C.c_int32),
        ("order", C.c_int32),
        ("nsub", C.c_int32),
        ("precision", C.c_int32),
        ("safety", C.c_double),
        ("t0", C.c_double),
        ("t1", C.c_double),
        ("dt", C.c_double),
        ("q2m", C.c_double),
        ("m", C.c_double),
        ("savestepinterval", C.c_int64),
        ("maxiters", C.c_int64),
        ("save_start", C.c_int32),
        ("save_end", C.c_int32),
        ("save_everystep", C.c_int32),
        ("save_fields", C.c_int32),
        ("term", TermDesc),
        ("step_cap", C.c_int64),
        ("schedule", C.c_int32),
        ("block", C.c_int32),
        ("budget_s", C.c_double),
        ("save_work", C.c_int32),
        ("particles_per_thread", C.c_int32),
    ]


class GCDesc(C.Structure):
    _fields_ = [
        ("alg", C.c_int32),
        ("precision", C.c_int32),
        ("t0", C.c_double),
        ("t1", C.c_double),
        ("dt", C.c_double),
        ("dt_given", C.c_int32),
        ("reserved", C.c_int32),
        ("q", C.c_double),
        ("q2m", C.c_double),
        ("mu", C.c_double),
        ("abstol", C.c_double),
        ("reltol", C.c_double),
        ("savestepinterval", C.c_int64),
        ("maxiters", C.c_int64),
        ("save_start", C.c_int32),
        ("save_end", C.c_int32),
        ("save_everystep", C.c_int32),
        ("save_fields", C.c_int32),
        ("term", TermDesc),
        ("block", C.c_int32),
        ("reserved2", C.c_int32),
        ("budget_s", C.c_double),
        ("save_work", C.c_int32),
        ("reserved3", C.c_int32),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("block", C.c_int32),
        ("schedule", C.c_int32),
        ("ms", C.c_double),
        ("ms_default", C.c_double),
        ("candidates", C.c_int32),
        ("particles_per_thread", C.c_int32),
    ]


class HybridDesc(C.Structure):
    _fields_ = [
        ("t0", C.c_double),
        ("t1", C.c_double),
        ("q2m", C.c_double),
        ("m", C.c_double),
        ("threshold_gc_to_fo", C.c_double),
        ("threshold_fo_to_gc", C.c_double),
        ("dtmin", C.c_double),
        ("dtmax", C.c_double),
        ("safety_fo", C.c_double),
        ("abstol", C.c_double),
        ("reltol", C.c_double),
        ("maxiters", C.c_int64),
        ("check_interval", C.c_int64),
        ("savestepinterval", C.c_int64),
        ("adiabaticity", C.c_int32),
        ("save_adiabaticity", C.c_int32),
        ("save_start", C.c_int32),
        ("save_end", C.c_int32),
        ("save_everystep", C.c_int32),
        ("block", C.c_int32),
        ("term", TermDesc),
        ("budget_s", C.c_double),
    ]


class Surface(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("point", _D3),
        ("normal", _D3),
        ("radius", C.c_double),
    ]


class PointsDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("want", C.c_int32),
        ("stride", C.c_int32),
        ("reserved", C.c_int32),
        ("q2m", C.c_double),
        ("m", C.c_double),
        ("q", C.c_double),
        ("mu", C.c_double),
    ]


class AdjDesc(C.Structure):
    _fields_ = [
        ("run", RunDesc),
        ("checkpoint_every", C.c_int64),
    ]


_P = C.c_void_p
_DP = C.POINTER(C.c_double)

# (name, restype, argtypes) of every symbol include/tp_abi.h declares
SIGNATURES = [
    ("tp_abi_version", C.c_int, []),
    ("tp_ctx_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("tp_ctx_destroy", None, [_P]),
    ("tp_last_error", C.c_char_p, [_P]),
    ("tp_field_create", C.c_int, [_P, C.POINTER(FieldDesc), C.POINTER(_P)]),
    ("tp_field_destroy", None, [_P]),
    ("tp_boris_run", C.c_int, [_P, C.POINTER(RunDesc), _P, _P, _P, _P, _P, C.c_int64, C.POINTER(_P)]),
    ("tp_boris_slots", C.c_int, [C.POINTER(RunDesc), _P, _P, C.c_int64, C.POINTER(C.c_int64)]),
    ("tp_boris_run_host", C.c_int,
     [_P, C.POINTER(RunDesc), _P, _P, _P, _P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P,
      C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    ("tp_boris_run_device", C.c_int,
     [_P, C.POINTER(RunDesc), _P, _P, _P, _P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P, _P, _P]),
    ("tp_gc_run", C.c_int, [_P, C.POINTER(GCDesc), _P, _P, _P, _P, _P, _P, _P, _P, C.c_int64, C.POINTER(_P)]),
    ("tp_gc_prepare", C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_double, C.c_double, C.c_double, _P, _P]),
    ("tp_gc_to_full", C.c_int, [_P, _P, _P, _P, _P, C.c_int64, C.c_double, C.c_double, C.c_double, _P, C.c_double,
                                _P]),
    ("tp_result_info", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    ("tp_result_copy", C.c_int, [_P, _P, _P, _P, _P, _P]),
    ("tp_result_elapsed_ms", C.c_int, [_P, _DP]),
    ("tp_result_destroy", None, [_P]),
    ("tp_pack_results_device_noalloc", C.c_int,
     [_P, _P, _P, _P, C.c_int64, C.c_int64, C.c_int32, _P, _P, _P, _P]),
    ("tp_field_update", C.c_int, [_P, _P]),
    ("tp_eval_points", C.c_int, [_P, C.POINTER(PointsDesc), _P, _P, _P, _P, C.c_int64, _P]),
    ("tp_eval_points_params", C.c_int, [_P, C.POINTER(PointsDesc), _P, _P, _P, _P, _P, _P, _P, _P, C.c_int64, _P]),
    ("tp_detect_fluxes", C.c_int,
     [_P, _P, _P, C.c_int32, _P, C.c_int64, C.POINTER(Surface), C.c_int32, _P, C.c_double, _P, _P]),
    ("tp_detect_crossings", C.c_int,
     [_P, _P, _P, C.c_int32, _P, C.c_int64, C.POINTER(Surface), C.c_int32, _P, C.c_double, _P, _P]),
    ("tp_detect_first_crossing", C.c_int, [_P, _P, _P, C.c_int32, _P, C.c_int64, C.POINTER(Surface), _P]),
    ("tp_hybrid_run", C.c_int, [_P, C.POINTER(HybridDesc), _P, _P, _P, C.c_int64, C.POINTER(_P), C.POINTER(_P)]),
    ("tp_autotune", C.c_int, [_P, C.POINTER(RunDesc), _P, _P, _P, C.c_int64, C.c_int64, C.POINTER(TuneResult)]),
    ("tp_boris_graph_create", C.c_int,
     [_P, C.POINTER(RunDesc), _P, _P, _P, _P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    ("tp_graph_launch", C.c_int, [_P, _P]),
    ("tp_graph_destroy", None, [_P]),
    ("tp_adjoint_forward", C.c_int, [_P, C.POINTER(AdjDesc), _P, _P, _P, C.c_int64, _P, C.POINTER(_P)]),
    ("tp_adjoint_backward", C.c_int, [_P, _P, _P, _P, _P, _P]),
    ("tp_adjoint_forward_device", C.c_int,
     [_P, C.POINTER(AdjDesc), _P, _P, _P, C.c_int64, _P, C.POINTER(_P), _P]),
    ("tp_adjoint_backward_device", C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    ("tp_tape_rerun_device", C.c_int, [_P, _P, _P, _P]),
    ("tp_tape_info", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("tp_tape_segments", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("tp_tape_destroy", None, [_P]),
]

# static scratch limit of tp_pack_results_device_noalloc (include/tp_abi.h)
TP_NOALLOC_MAX_TRAJECTORIES = 1048576

_lib = None


def load_library(path: Path | None = None) -> C.CDLL:
    """Load libtpb200.so (built in-tree by build_ext.py) and bind its symbols."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python testparticle.jl_b200/build_ext.py` "
            "(the B200 library has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.tp_abi_version() != TP_ABI_VERSION:
        raise ImportError("libtpb200.so ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return [s[0] for s in SIGNATURES]
