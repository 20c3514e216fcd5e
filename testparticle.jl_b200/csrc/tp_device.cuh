// tp_device.cuh -- device-side types shared by the push kernels.
//
// Field evaluation for the kinds of include/tp_abi.h, the termination
// predicate, and the launch argument block.  Everything here is plain CUDA C++
// for sm_100a; there is no contraction (GEMM) anywhere in this path, so no
// tensor-core code: the kernels are FP64/FP32-pipe or L2-gather bound.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/tp_abi.h"

namespace tpb {

// ------------------------------------------------------------------ fields
// One field as the kernels see it.  Grid data lives in a per-node table
// (4 values per node, the 4th is padding) so that a corner is one aligned
// 16-byte (float) or 32-byte (double) load.  When E and B are grids on the
// same geometry the runtime builds one interleaved table (E then B per node,
// 32 bytes per node in float) so that each corner of a particle-step is a
// single 32-byte sector.
struct DevField {
    int32_t kind;
    int32_t bc;
    int32_t f64;      // grid table holds doubles
    int32_t pad0;
    double v[3];      // uniform value / affine constant
    double J[9];      // affine Jacobian (row-major)
    double rate[3];   // affine d/dt
    double m[3];      // dipole moment
    double c[3];      // dipole centre
    double coef;      // dipole mu0/4pi
    int32_t n[3];
    int32_t pad1;
    double x0[3];
    double inv_dx[3];
    double L[3];      // periodic length n*dx
    float x0f[3];     // float copies for the FP32C kernels
    float dxf[3];
    float idxf[3];
    float vf[3];      // uniform value / affine constant (float)
    float Jf[9];
    float ratef[3];
    float mf[3];
    float cf[3];
    float coeff;
    float mhatf[3];   // dipole: unit moment and K = coef * |m| (keeps float
    float Kf;         //   intermediates normal: coef / r^5 alone underflows)
    const void* tab;  // per-node table: float4 / double4 per node (x,y,z,0)
    const float4* tab32;  // float table for the FP32C kernels (same as tab for float data)
    // grids off the trilinear uniform Cartesian 3-D fast path (grid_general.cuh)
    int32_t general;  // 1: order, geometry, dimension or axes differ from the fast path
    int32_t order;    // TP_ORDER_*
    int32_t geom;     // TP_GRID_*
    int32_t dir;      // 1-D interpolant: the coordinate axis 0 reads
    int32_t abc[3];   // per-axis boundary (TP_BC_*)
    int32_t ndim;
    const double* ax[3];  // device node coordinates of non-uniform axes, else null
    double Q[27];     // quadratic field: Q[9 i + 3 j + k] x_j x_k
    // time series (LazyTimeInterpolator): snapshots at sorted times
    const DevField* snaps;
    const double* ts;
    int32_t nts;
    int32_t pad2;
    // a copy of this descriptor in device memory: the out-of-line evaluators
    // of the general grids, quadratic fields and series take it, so a call
    // passes a global pointer instead of copying the kernel-parameter struct
    // to local memory
    const DevField* self;
};

// QUADRATIC field value in float64, in the order of the CPU restatement:
// F_i = ((v_i + ((J_i0 x + J_i1 y) + J_i2 z)) + q_i) + rate_i t with
// q_i = (x (Q_i0. x) + y (Q_i1. x)) + z (Q_i2. x), Q_ij. x = (Q_ij0 x + Q_ij1 y) + Q_ij2 z
__device__ __forceinline__ void quad_eval(const DevField& f, double x, double y, double z, double t,
                                          double o[3]) {
    for (int i = 0; i < 3; ++i) {
        const double* J = f.J + 3 * i;
        const double* Q = f.Q + 9 * i;
        double lin = (J[0] * x + J[1] * y) + J[2] * z;
        double qx = (Q[0] * x + Q[1] * y) + Q[2] * z;
        double qy = (Q[3] * x + Q[4] * y) + Q[5] * z;
        double qz = (Q[6] * x + Q[7] * y) + Q[8] * z;
        double q = (x * qx + y * qy) + z * qz;
        o[i] = ((f.v[i] + lin) + q) + f.rate[i] * t;
    }
}

struct DevFields {
    DevField E, B;
    const void* eb;   // interleaved table (E xyz0, B xyz0) per node, or null
    const float4* eb32;   // float interleaved table for the FP32C kernels
    int32_t eb_f64;
    int32_t pad;
    // E and B on one periodic, uniform, Cartesian 3-D grid of order 3: their
    // float interleaved table (the warp-cooperative FP32C kernel), else null
    const float4* ebc32;
};

// Termination predicate (the reference's isoutside, as flags).
struct DevTerm {
    int32_t flags;
    int32_t pad;
    double rmin, rmax;
    double lo[3], hi[3];
    double tmax;
};

// Field configurations a kernel is specialised for (keeps register use down):
//   FK_ANALYTIC  E and B analytic (zero / uniform / affine / dipole)
//   FK_EBGRID    E and B grids on one geometry, interleaved table
//   FK_GENERIC   anything else (separate grids, grid + analytic)
//   FK_GENGRID   at least one grid off the trilinear uniform Cartesian path
//                (order 0 / 3, rectilinear, spherical, 1-D / 2-D)
enum { FK_ANALYTIC = 0, FK_EBGRID = 1, FK_GENERIC = 2, FK_GENGRID = 3 };

__host__ __device__ __forceinline__ int field_config_of(const DevFields& f) {
    if ((f.E.kind == TP_FIELD_GRID && f.E.general) || (f.B.kind == TP_FIELD_GRID && f.B.general) ||
        f.E.kind == TP_FIELD_SERIES || f.B.kind == TP_FIELD_SERIES)
        return FK_GENGRID;
    if (f.E.kind == TP_FIELD_QUADRATIC || f.B.kind == TP_FIELD_QUADRATIC) return FK_GENERIC;
    if (f.eb && !f.eb_f64) return FK_EBGRID;  // float interleaved table
    if (f.E.kind != TP_FIELD_GRID && f.B.kind != TP_FIELD_GRID) return FK_ANALYTIC;
    return FK_GENERIC;
}

// ------------------------------------------------------------------ launch
struct BorisArgs {
    DevFields f;
    DevTerm term;
    int32_t alg, order, nsub, save_fields;
    int32_t save_start, save_end, save_everystep, use_queue;
    double safety, t0, t1, dt, q2m, m;
    int64_t ssi, maxiters, step_cap;
    int64_t n, nslots;
    const double* u0;     // 6 x n (column-major)
    const double* dt_i;   // optional
    const double* tend_i; // optional
    double* t_out;        // nslots x n
    double* u_out;        // nslots x W x n
    int32_t* nsaved;
    int8_t* retcode;
    int64_t* nsteps;
    int32_t* status;      // device: first error code
    unsigned long long* queue;  // persistent-schedule work counter
    uint64_t budget_ns;
    // FP32C only: per axis, wrap positions into the periodic box
    int32_t wrap[3];
    int32_t save_work;    // work rates appended to every save (width + 4)
    double wrapL[3], wrap0[3];
    int32_t ppt;          // particles per thread of the fixed-step kernels (1 or 2)
    int32_t pad_ppt;
    // optional processing order: the k-th particle a kernel takes is perm[k]
    // (a cell ordering of the initial positions in gridded fields, so that
    // the lanes of a warp gather neighbouring nodes); null = 0, 1, 2, ...
    const int32_t* perm;
    // optional completion counts: once particle i's outputs are written it
    // adds 1 to done[i / done_chunk], so a host can copy out finished index
    // ranges while the kernel runs; null = off
    int32_t* done;
    int64_t done_chunk;
};

// particle i's outputs are final: publish them, then count the particle
__device__ __forceinline__ void particle_done(const BorisArgs& a, int64_t i) {
    if (a.done) {
        __threadfence_system();
        atomicAdd(a.done + i / a.done_chunk, 1);
    }
}

// the particle taken k-th under the run's processing order (k < n)
__device__ __forceinline__ int64_t take_particle(const BorisArgs& a, int64_t k) {
    return (a.perm && k < a.n) ? (int64_t)__ldg(a.perm + k) : k;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void set_status(int32_t* status, int32_t code) {
    if (status) atomicCAS(status, 0, code);
}

// Julia round(Int, x): ties to even (rint in the default rounding mode)
__device__ __forceinline__ int64_t jl_round(double x) { return (int64_t)rint(x); }

// _calculate_nout, src/boris/boris.jl:383-403
__device__ __forceinline__ int64_t calc_nout(int64_t nt, int64_t ssi, bool ss, bool se, bool sev) {
    int64_t nout = 0;
    if (ss) nout += 1;
    if (sev) {
        int64_t steps = nt / ssi;
        bool last_is_step = (nt > 0) && (nt % ssi == 0);
        nout += steps;
        if (!se && last_is_step) nout -= 1;
        if (se && !last_is_step) nout += 1;
    } else if (se) {
        nout += 1;
    }
    return nout;
}

}  // namespace tpb

// Largest block a push kernel is compiled for, per field configuration: it
// caps the register allocation at 65536 / TPB_MAXT(FK) per thread.  The
// interleaved-grid kernels are gather-latency bound, so they take 384 (<= 170
// registers: three 128-thread blocks per SM); at 512 the float64 one spills
// 340 bytes per thread and measured 7 % slower on the 128^3 gridded
// workload (1.93e10 against 2.07e10 particle-steps/s, four blocks per SM
// instead of three), and the FP32C one spills 70-110 bytes and measured
// 8 % slower at 448 or 512 (2.77e10 against 3.02e10): spills add traffic to
// the L1 path that bounds it.  The analytic-field kernels are latency bound
// on float64 dependency chains and launch up to 512 threads: the float64
// multistep and adaptive pushes in the dipole measured 15 % faster than at
// 256 (the fixed-step and adaptive ones are compiled for larger blocks
// still, below).  The others take 256.
#define TPB_MAXT(FK) ((FK) == FK_EBGRID ? 384 : ((FK) == FK_ANALYTIC ? 512 : 256))

// Register cap of the one-particle-per-thread fixed-step kernels (k_fixed32c,
// k_fixed64).  In analytic fields they are compiled for blocks of up to 768
// threads (<= 80 registers per thread, six 128-thread blocks per SM) although
// launches stay at or below TPB_MAXT: the extra resident warps hide the
// float64 dependency latency that bounds them, and outweigh the 40-150 bytes
// of spills this costs.  On the dipole ensemble (MultistepBoris4(2), 1e6 x 1e4)
// the FP32C push measured 7.50e10 -> 7.93e10 particle-steps/s (caps of 640,
// 896 and 1024 threads: 7.69e10, 7.64e10, 7.58e10) and the float64 push
// 2.71e10 -> 2.88e10 (640: 2.80e10).
#define TPB_FIXED_BOUND(FK) ((FK) == FK_ANALYTIC ? 768 : TPB_MAXT(FK))

// The same for the adaptive kernels in analytic fields (AdaptiveBoris(0.1)
// on the dipole ensemble, 1e6 particles, cap 1e4 steps): FP32C at 640
// threads (<= 96 registers) 3.39e10 -> 3.57e10 particle-steps/s (768:
// 3.54e10), float64 at 768 (<= 80) 2.32e10 -> 2.44e10 (640: 2.42e10).
#define TPB_ADAPTIVE32_BOUND(FK) ((FK) == FK_ANALYTIC ? 640 : TPB_MAXT(FK))
#define TPB_ADAPTIVE64_BOUND(FK) ((FK) == FK_ANALYTIC ? 768 : TPB_MAXT(FK))
