"""TestParticle B200: the particle-push hot path of TestParticle.jl on one B200.

Host-side mirror of the reference API (prepare, TraceProblem, TraceGCProblem,
solve with Boris / MultistepBoris / AdaptiveBoris / :rk4 / :rk45) over the C
ABI of libtpb200.so (include/tp_abi.h).  All trajectories are computed by the
CUDA kernels of csrc/; a missing library raises ImportError.

This directory is imported under the module name `testparticle_b200`.
"""
from __future__ import annotations

from . import _abi, workloads
from .constants import (BMoment_Earth, Electron, Ion, MU0_OVER_4PI, Proton, Re, Species, SpeciesDict,
                        c, eV, kB, me, mi, mu0, qe, qi)
from .fields import (AffineField, CartesianGrid, ClampExtrap, DipoleField, FieldInterpolator, FillExtrap,
                     LazyTimeInterpolator, PeriodicBC, QuadraticField, RectilinearGrid, StructuredGrid, UniformField, WrapExtrap, ZeroField,
                     build_interpolator)
from .problems import (AdaptiveBoris, AdaptiveHybrid, AdaptiveMultistepBoris, Boris, EnsembleB200, EnsembleContext,
                       MultistepBoris, MultistepBoris2, MultistepBoris4, MultistepBoris6, Terminate,
                       TerminateBox, TerminateNaN, TerminateShell, TerminateTime, TraceGCProblem,
                       TraceHybridProblem, TraceProblem, prepare, remake)
from .detectors import (Disk, Plane, Sphere, get_first_crossing, get_particle_crossings, get_particle_flux,
                        get_particle_fluxes)
from .postprocess import get_fields, get_work
from .runtime import AdjointGrads, ArgumentError, Context, DeviceError, Tape
from .solution import EnsembleSolution, TraceSolution
from .solve import (AdjointPlan, BorisPlan, GCPlan, HybridPlan, adjoint_solve, full_to_gc, gc_to_full, plan_adjoint,
                    plan_boris, plan_gc, plan_hybrid, prepare_gc, solve)
from .utility import energy2velocity, get_gyrofrequency, get_gyroperiod, get_gyroradius, get_perp_vector, sph2cart

__version__ = "0.1.0"
