"""CPU checks of the boundary and the host logic (no kernel is launched).

* libtpb200.so loads and exports every function include/tp_abi.h declares;
* the host-side sizing (tp_boris_slots) equals the reference's nout rule as
  restated by the oracle (src/boris/boris.jl:383-403);
* the Python mirror builds descriptors, validates arguments and rejects
  what cannot run on the device;
* the seeded workload generators are deterministic.
"""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "tp_abi.h"


def _declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(tp_\w+)\s*\(", text, re.M)))


def test_header_matches_binding_table(tp):
    assert _declared() == sorted(tp._abi.declared_symbols())


def test_library_loads_and_exports_every_symbol(tp):
    lib = tp._abi.load_library()
    for name in _declared():
        assert hasattr(lib, name)
    out = subprocess.run(["nm", "-D", "--defined-only", str(tp._abi.LIB_PATH)], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (tp_\w+)", out))
    assert set(_declared()) <= exported
    assert lib.tp_abi_version() == tp._abi.TP_ABI_VERSION


def test_ctx_create_without_gpu_fails_cleanly(tp):
    lib = tp._abi.load_library()
    h = C.c_void_p()
    code = lib.tp_ctx_create(0, C.byref(h))
    assert code in (tp._abi.TP_OK, tp._abi.TP_E_CUDA)
    if code == tp._abi.TP_OK:
        lib.tp_ctx_destroy(h)
    assert lib.tp_ctx_create(0, None) == tp._abi.TP_E_ARG


@pytest.mark.parametrize("ssi", [1, 3, 7, 10, 100, 1000])
@pytest.mark.parametrize("flags", [(1, 1, 1), (0, 1, 0), (1, 1, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1)])
def test_slot_count_equals_reference_nout(tp, orc, ssi, flags):
    lib = tp._abi.load_library()
    ss, se, sev = flags
    for nt in (0, 1, 9, 10, 11, 999, 1000, 1001):
        d = tp._abi.RunDesc()
        d.alg = tp._abi.TP_ALG_BORIS
        d.t0, d.t1, d.dt = 0.0, nt * 0.5, 0.5
        d.savestepinterval, d.maxiters = ssi, 10**6
        d.save_start, d.save_end, d.save_everystep = ss, se, sev
        ns = C.c_int64()
        assert lib.tp_boris_slots(C.byref(d), None, None, 1, C.byref(ns)) == 0
        assert ns.value == orc.boris_counts(0.0, nt * 0.5, 0.5, 10**6, ssi, bool(ss), bool(se), bool(sev))[1]


def test_slot_count_rejects_reference_argument_errors(tp):
    lib = tp._abi.load_library()
    d = tp._abi.RunDesc()
    d.alg, d.t0, d.t1, d.dt, d.savestepinterval, d.maxiters = 0, 0.0, 1e-9, 1e-11, 1, 50
    ns = C.c_int64()
    assert lib.tp_boris_slots(C.byref(d), None, None, 1, C.byref(ns)) == tp._abi.TP_E_ARG  # nt > maxiters
    d.maxiters, d.dt = 10**6, np.finfo(float).eps
    assert lib.tp_boris_slots(C.byref(d), None, None, 1, C.byref(ns)) == tp._abi.TP_E_ARG  # dt < 10 eps


def test_plan_descriptor(tp):
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 1e-8)), species=tp.Proton)
    prob = tp.TraceProblem(np.zeros((6, 5)), (0.0, 1.0), param)
    p = tp.plan_boris(prob, tp.MultistepBoris4(2), tp.EnsembleB200(precision="fp32c"), dt=0.01,
                      savestepinterval=7, isoutside=tp.TerminateShell(1.0, 2.0) | tp.TerminateNaN())
    d = p.desc
    assert (d.alg, d.order, d.nsub, d.precision) == (tp._abi.TP_ALG_MULTISTEP, 4, 2, tp._abi.TP_PREC_FP32C)
    assert d.q2m == tp.qi / tp.mi and d.savestepinterval == 7 and d.maxiters == 1_000_000
    assert d.term.flags == tp._abi.TP_TERM_SHELL | tp._abi.TP_TERM_NAN
    assert (d.term.rmin, d.term.rmax) == (1.0, 2.0)
    assert p.u0.shape == (5, 6)


def test_prob_func_builds_table(tp):
    param = tp.prepare(tp.ZeroField(), tp.UniformField((0.0, 0.0, 0.01)), species=tp.Electron)

    def pf(prob, ctx):
        u = list(prob.u0)
        u[4] = ctx.sim_id * 1.0e5
        return tp.remake(prob, u0=u)

    prob = tp.TraceProblem([0.0, 0.0, 0.0, 0.0, 1.0e5, 0.0], (0.0, 3e-8), param, prob_func=pf)
    p = tp.plan_boris(prob, tp.Boris(), dt=3e-11, trajectories=3)
    assert list(p.u0[:, 4]) == [1e5, 2e5, 3e5]


def test_unsupported_inputs_raise(tp):
    with pytest.raises(NotImplementedError):
        tp.prepare(lambda x: (0, 0, 1), lambda x: (0, 0, 1))
    with pytest.raises(NotImplementedError):
        tp.plan_boris(tp.TraceProblem(np.zeros(6), (0, 1), tp.prepare(tp.ZeroField(), tp.ZeroField())),
                      tp.Boris(), dt=0.1, isoutside=lambda u, p, t: False)
    with pytest.raises(ValueError):
        tp.MultistepBoris(3)
    # interpolation.jl:145-146,246-248: unsupported orders and cubic rectilinear grids
    with pytest.raises(ValueError):
        tp.build_interpolator(np.zeros((3, 4, 4, 4)), np.arange(4.0), np.arange(4.0), np.arange(4.0), 2)
    with pytest.raises(ValueError):
        tp.build_interpolator(tp.RectilinearGrid, np.zeros((3, 4, 4, 4)), [0, 1, 3, 4.0], np.arange(4.0),
                              np.arange(4.0), 3)
    with pytest.raises(ValueError):   # StructuredGrid assertions (:270-280)
        tp.build_interpolator(tp.StructuredGrid, np.zeros((3, 4, 4, 4)), np.arange(4.0),
                              np.linspace(0, 4.0, 4), np.linspace(0, 6.0, 4))


def test_grid_field_layout_is_julia_column_major(tp):
    A = np.arange(3 * 2 * 3 * 4, dtype=np.float32).reshape(3, 2, 3, 4)
    f = tp.build_interpolator(A, [0.0, 1.0], [0.0, 1.0, 2.0], [0.0, 1.0, 2.0, 3.0])
    flat = np.frombuffer(f.data.tobytes(order="A"), dtype=np.float32)
    # component c of node (i, j, k) sits at c + 3*(i + nx*(j + ny*k))
    for c, i, j, k in [(0, 0, 0, 0), (2, 1, 0, 0), (1, 0, 2, 1), (2, 1, 2, 3)]:
        assert flat[c + 3 * (i + 2 * (j + 3 * k))] == A[c, i, j, k]


def test_workloads_are_deterministic(tp):
    a = tp.workloads.config1(16)
    b = tp.workloads.config1(16)
    assert np.array_equal(a.u0, b.u0)
    r = tp.workloads.SplitMix64(1)
    # SplitMix64 reference outputs for seed 1 (first two values of the published generator)
    assert list(r.next_u64(2)) == [0x910A2DEC89025CC1, 0xBEEB8DA1658EEC67]
    w = tp.workloads.config3(64, nt=100)
    assert np.all(np.abs(w.u0[2]) == 0.0)
    assert np.allclose(w.tend, 100 * w.dt)
