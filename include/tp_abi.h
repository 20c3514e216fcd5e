/*
 * tp_abi.h -- C ABI of the B200 particle-push library (libtpb200.so).
 *
 * The reference (TestParticle.jl v0.23.2) is pure Julia and has no FFI of its
 * own; its hot path is entered through the ensemble-algorithm dispatch
 *
 *     TestParticle.solve(prob, alg, ensemblealg; dt, savestepinterval, ...)
 *       -> _solve(::EnsembleAlg, prob::TraceProblem, alg::AbstractBoris, ...)
 *                                        (src/boris/boris.jl:88-114,137-318)
 *       -> _solve_adaptive(::EnsembleAlg, ...)   (src/boris/adaptive_boris.jl:21-139)
 *       -> _solve(::EnsembleAlg, prob::TraceGCProblem, ...)
 *                                        (src/gc/gc_solver.jl:59-161)
 *
 * A Julia package binds the entry points below with `ccall` from new
 * `_solve(::EnsembleB200, ...)` methods, so a user call such as
 * `TestParticle.solve(prob, Boris(), EnsembleB200(); dt, savestepinterval,
 * trajectories)` returns the reference's EnsembleSolution layout.  Python
 * binds the same symbols with ctypes.
 *
 * Conventions
 *  - Every function returns an int status: TP_OK (0) or a negative TP_E_*.
 *    TP_E_ARG corresponds to the reference's ArgumentError
 *    (src/boris/boris.jl:349-356, src/types.jl:71-73); the others to
 *    ErrorException.  The text of the last error of a context is returned by
 *    tp_last_error().  No entry point aborts or traps.
 *  - Input pointers are borrowed for the duration of the call.  Grid data
 *    (host or device memory) is copied to the device by tp_field_create().
 *    Results are owned by a tp_result until tp_result_destroy().
 *  - Calls on one context are synchronous and must come from one thread at a
 *    time.  Device entry points (suffix _device) are asynchronous on the
 *    stream they are given.
 *  - Particle state tables are 6 x N float64, column-major (Julia's layout of
 *    a Matrix{Float64}(6, N)): element c of particle i is u0[6*i + c].
 */
#ifndef TP_ABI_H
#define TP_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TP_ABI_VERSION 3

/* ---- status codes ------------------------------------------------------ */
enum {
    TP_OK = 0,
    TP_E_ARG = -1,         /* invalid argument: reference ArgumentError     */
    TP_E_CUDA = -2,        /* CUDA runtime error                             */
    TP_E_TIMEOUT = -3,     /* device loop exceeded its wall-clock budget     */
    TP_E_NOMEM = -4,       /* device or host allocation failed               */
    TP_E_UNSUPPORTED = -5, /* field / algorithm combination not implemented  */
    TP_E_OVERFLOW = -6     /* a particle produced more saves than slots      */
};

/* ---- per-trajectory return codes (SciMLBase.ReturnCode subset) --------- */
enum {
    TP_RET_DEFAULT = 0,
    TP_RET_SUCCESS = 1,    /* ReturnCode.Success    */
    TP_RET_TERMINATED = 2, /* ReturnCode.Terminated */
    TP_RET_MAXITERS = 3    /* ReturnCode.MaxIters   */
};

/* ---- fields --------------------------------------------------------------
 * The reference accepts any Julia callable F(x, t) as a field.  Callables
 * cannot cross a C ABI, so a field is described by one of these kinds:
 *   ZERO     ZeroField()                         (src/utility/zero.jl:35-51)
 *   UNIFORM  F(x,t) = value
 *   AFFINE   F(x,t) = value + jac * x + rate * t  (uniform, gradient and
 *            linearly time-varying fields of the reference tests)
 *   DIPOLE   F(x) = coef * (3 (m.rhat) rhat - m) / |x - center|^3
 *            (the Magnetostatics.Dipole field of test/test_gc.jl:180)
 *   QUADRATIC  F_i(x,t) = value_i + sum_j jac_ij x_j + sum_jk quad_ijk x_j x_k
 *            + rate_i t (the quadratic test fields of the reference, e.g.
 *            the magnetic bottle of test/test_hybrid.jl:61-68)
 *   SERIES   LazyTimeInterpolator(times, loader) (src/utility/interpolation.jl:
 *            337-430): snapshot fields at sorted times, blended linearly in
 *            time, (1 - w) F_k(x) + w F_{k+1}(x), and clamped to the first /
 *            last snapshot outside [times[0], times[n-1]].  Every snapshot
 *            is uploaded and stays resident on the device.
 *   GRID     interpolation of a (3, nx, ny, nz) column-major array:
 *            build_interpolator(gridtype, A, grids..., order, bc)
 *            (src/utility/interpolation.jl:119-311).  The default (a zeroed
 *            descriptor tail) is trilinear on a uniform Cartesian grid; the
 *            tail fields below select the order (0 / 1 / 3), rectilinear
 *            axes, spherical geometry and 1-D / 2-D interpolants.          */
enum {
    TP_FIELD_ZERO = 0,
    TP_FIELD_UNIFORM = 1,
    TP_FIELD_AFFINE = 2,
    TP_FIELD_DIPOLE = 3,
    TP_FIELD_GRID = 4,
    TP_FIELD_QUADRATIC = 5,
    TP_FIELD_SERIES = 6
};

/* grid boundary handling (FastInterpolations FillExtrap(NaN), ClampExtrap(),
 * PeriodicBC(endpoint=:exclusive) / WrapExtrap() with period L = n * dx,
 * PeriodicBC(endpoint=:inclusive) with period L = (n - 1) * dx: the last
 * node repeats the first)                                                   */
enum {
    TP_BC_FILL_NAN = 0,
    TP_BC_CLAMP = 1,
    TP_BC_PERIODIC = 2,
    TP_BC_PERIODIC_INCLUSIVE = 3
};

/* interpolation order of a grid (build_interpolator's `order`):
 *   LINEAR    order 1, linear_interp (the default)
 *   CONSTANT  order 0, constant_interp: the nearest node
 *   CUBIC     order 3, cardinal_interp: local cubic Hermite (Catmull-Rom)
 *             on uniform axes                                              */
enum {
    TP_ORDER_LINEAR = 0,
    TP_ORDER_CONSTANT = 1,
    TP_ORDER_CUBIC = 2
};

/* grid geometry:
 *   CARTESIAN  axes x, y, z (CartesianGrid, or RectilinearGrid when node
 *              coordinates are given per axis)
 *   SPHERICAL  axes r, theta, phi (StructuredGrid,
 *              SphericalFieldInterpolator, interpolation.jl:97-117,260-284):
 *              the point is converted with cart2sph, r and theta fill NaN
 *              outside the grid, phi is periodic (inclusive), and the
 *              interpolated (v_r, v_theta, v_phi) is returned in Cartesian
 *              components (sph2cartvec, src/utility/utility.jl:82-89)      */
enum {
    TP_GRID_CARTESIAN = 0,
    TP_GRID_SPHERICAL = 1,
    TP_GRID_SPHERICAL_SCALAR = 2 /* spherical grid of a scalar carried in
                                    component 0: no basis conversion      */
};

enum { TP_DTYPE_F32 = 0, TP_DTYPE_F64 = 1 };

typedef struct tp_field_desc {
    int32_t kind;        /* TP_FIELD_*                                      */
    int32_t bc;          /* GRID: TP_BC_*                                   */
    int32_t dtype;       /* GRID: TP_DTYPE_* of data                        */
    int32_t reserved;
    double value[3];     /* UNIFORM value; AFFINE constant term             */
    double jac[9];       /* AFFINE: d F_i / d x_j, row-major                */
    double rate[3];      /* AFFINE: d F / d t                               */
    double moment[3];    /* DIPOLE: magnetic moment [A m^2]                 */
    double center[3];    /* DIPOLE: position of the dipole                  */
    double coef;         /* DIPOLE: mu0 / 4pi                               */
    int64_t n[3];        /* GRID: nodes along x, y, z (each >= 2)           */
    double origin[3];    /* GRID: coordinate of node (0,0,0)                */
    double spacing[3];   /* GRID: node spacing (> 0)                        */
    const void* data;    /* GRID: host pointer, 3*nx*ny*nz values, (3,nx,ny,nz)
                            column-major: component c of node (i,j,k) is at
                            c + 3*(i + nx*(j + ny*k))                       */
    /* GRID tail (all zero: trilinear, uniform Cartesian, 3-D)              */
    int32_t order;       /* TP_ORDER_*                                      */
    int32_t geometry;    /* TP_GRID_*                                       */
    int32_t ndim;        /* CARTESIAN: 1, 2 or 3 (0 = 3): FieldInterpolator1D
                            / 2D / 3D; unused axes have n = 1               */
    int32_t dir;         /* ndim 1: the coordinate (0, 1, 2) it reads       */
    const double* axis[3]; /* per-axis node coordinates (n[a] strictly
                            increasing values, host memory), or NULL for the
                            uniform axis origin + k * spacing.  Non-uniform
                            axes take LINEAR or CONSTANT order and FILL_NAN
                            or CLAMP boundaries.                            */
    double quad[27];     /* QUADRATIC: quad_ijk at [9 i + 3 j + k]          */
    int64_t nseries;     /* SERIES: number of snapshots (>= 1)              */
    const double* series_times;          /* SERIES: nseries sorted times    */
    const struct tp_field_desc* series;  /* SERIES: nseries snapshot
                            descriptors (any kind but SERIES)               */
} tp_field_desc;

/* ---- termination (the reference's `isoutside(u, p, t)` callback) --------
 * A Julia closure cannot cross the ABI; the common predicates are flags.
 * The predicate is evaluated where the reference calls isoutside:
 * src/boris/boris.jl:459, src/boris/adaptive_boris.jl:227,
 * src/gc/rk4_gc.jl:318, src/gc/rk45_gc.jl:128.                             */
enum {
    TP_TERM_SHELL = 1,   /* |x| < rmin or |x| > rmax                        */
    TP_TERM_BOX = 2,     /* any x_c < lo_c or x_c > hi_c                    */
    TP_TERM_NAN = 4,     /* any component of the state is NaN              */
    TP_TERM_TIME = 8     /* t > tmax                                        */
};

typedef struct tp_term_desc {
    int32_t flags;
    int32_t reserved;
    double rmin, rmax;
    double lo[3], hi[3];
    double tmax;
} tp_term_desc;

/* ---- full-orbit run ------------------------------------------------------ */
enum {
    TP_ALG_BORIS = 0,             /* Boris()                 boris.jl:480-557        */
    TP_ALG_MULTISTEP = 1,         /* MultistepBoris{N}(n)    multistep_boris.jl:65-142 */
    TP_ALG_ADAPTIVE = 2,          /* AdaptiveBoris(safety)   adaptive_boris.jl:145-266 */
    TP_ALG_ADAPTIVE_MULTISTEP = 3 /* AdaptiveMultistepBoris{N}(n, safety)             */
};

enum {
    TP_PREC_FP64 = 0,   /* plain float64, operation order of the reference   */
    TP_PREC_FP32C = 1   /* float32 push, positions as compensated float pairs */
};

enum {
    TP_SCHED_AUTO = 0,   /* library choice                                   */
    TP_SCHED_STATIC = 1, /* one thread per particle                          */
    TP_SCHED_QUEUE = 2   /* persistent kernel pulling particles from a queue */
};

typedef struct tp_run_desc {
    int32_t alg;             /* TP_ALG_*                                    */
    int32_t order;           /* multistep gyrophase order N: 2, 4 or 6      */
    int32_t nsub;            /* multistep subcycles n >= 1                  */
    int32_t precision;       /* TP_PREC_*                                   */
    double safety;           /* adaptive safety factor                      */
    double t0, t1;           /* tspan                                       */
    double dt;               /* fixed-step dt                               */
    double q2m, m;           /* p = (q2m, m, E, B, F) of prepare()          */
    int64_t savestepinterval;
    int64_t maxiters;        /* fixed step: nt > maxiters is TP_E_ARG       */
    int32_t save_start, save_end, save_everystep, save_fields;
    tp_term_desc term;
    int64_t step_cap;        /* adaptive: steps per particle, 0 = no cap    */
    int32_t schedule;        /* TP_SCHED_*                                  */
    int32_t block;           /* threads per block, 0 = tuned / default      */
    double budget_s;         /* device wall-clock budget, 0 = default 600 s */
    int32_t save_work;       /* append (P_par, P_fermi, P_grad, P_betatron)
                                to every save (boris.jl:405-440)            */
    int32_t particles_per_thread; /* fixed step, analytic fields: 1 or 2
                                particles advanced in lock step by each
                                thread; 0 = tuned / default (1)             */
} tp_run_desc;

/* ---- guiding-centre run ------------------------------------------------- */
enum { TP_GC_RK4 = 0, TP_GC_RK45 = 1 };
enum { TP_GC_PREC_FP64 = 0, TP_GC_PREC_FP32RHS = 1 };

typedef struct tp_gc_desc {
    int32_t alg;             /* TP_GC_RK4 (rk4_gc.jl) / TP_GC_RK45 (rk45_gc.jl)   */
    int32_t precision;       /* TP_GC_PREC_*                                     */
    double t0, t1;
    double dt;               /* RK4 step / RK45 initial step                     */
    int32_t dt_given;        /* 0: RK45 picks half a gyroperiod (rk45_gc.jl:82-99) */
    int32_t reserved;
    double q, q2m, mu;       /* p = (q, q2m, mu, E, B) of prepare_gc()          */
    double abstol, reltol;
    int64_t savestepinterval;
    int64_t maxiters;
    int32_t save_start, save_end, save_everystep, save_fields;
    tp_term_desc term;
    int32_t block;
    int32_t reserved2;
    double budget_s;
    int32_t save_work;       /* append the work rates (gc_solver.jl:233-248) */
    int32_t reserved3;
} tp_gc_desc;

typedef struct tp_ctx tp_ctx;
typedef struct tp_field tp_field;
typedef struct tp_result tp_result;

/* ---- library and context ------------------------------------------------- */
int tp_abi_version(void);
int tp_ctx_create(int device, tp_ctx** out);
void tp_ctx_destroy(tp_ctx* ctx);
const char* tp_last_error(const tp_ctx* ctx);

/* ---- fields --------------------------------------------------------------
 * Replaces prepare_field / build_interpolator (src/prepare.jl:86-104,
 * src/utility/interpolation.jl:217-235): the field is validated and any grid
 * is uploaded once.                                                         */
int tp_field_create(tp_ctx* ctx, const tp_field_desc* desc, tp_field** out);
void tp_field_destroy(tp_field* field);
/* Replace the node values of a grid field in place (same geometry and dtype;
 * `data` is host or device memory of the field's size).  The next solve sees
 * the new values; tapes recorded before the update must not be reused.  An
 * addition for optimisation loops over gridded fields (the reference rebuilds
 * the interpolator).                                                        */
int tp_field_update(tp_field* field, const void* data);

/* ---- adaptive hybrid guiding-centre / full-orbit solve --------------------
 * Replaces solve(::TraceHybridProblem, ::AdaptiveHybrid, ensemblealg)
 * (src/hybrid.jl:123-474): per particle, RK45 guiding-centre steps while the
 * adiabaticity parameter stays below threshold_gc_to_fo, Boris full-orbit
 * steps (dt = 2 pi safety_fo / (|q2m| |B|) clamped to [dtmin, dtmax]) until
 * it drops below threshold_fo_to_gc, checked every check_interval steps.
 * Saves are full-orbit states (x, v), 6 values.  The adiabaticity value and
 * mode of every check are returned in a second result of width 2 (value,
 * mode: 0 = GC, 1 = FO) when `adia` is not NULL.  Return codes follow the
 * reference: MaxIters when maxiters steps were taken, else Success; a step
 * whose error norm is NaN ends the trajectory with Terminated (the reference
 * would retry it forever).                                                  */
enum {
    TP_ADIA_CURVATURE = 0, /* epsilon = rho / R_c                            */
    TP_ADIA_GRADB = 1,     /* epsilon = rho / L_B, L_B = |B| / |grad|B||     */
    TP_ADIA_BOTH = 2,      /* max of the two                                 */
    TP_ADIA_JACOBIAN = 3   /* epsilon = rho ||JB||_F / |B|                   */
};

typedef struct tp_hybrid_desc {
    double t0, t1;
    double q2m, m;
    double threshold_gc_to_fo, threshold_fo_to_gc;
    double dtmin, dtmax, safety_fo;
    double abstol, reltol;
    int64_t maxiters;
    int64_t check_interval;
    int64_t savestepinterval;
    int32_t adiabaticity;     /* TP_ADIA_*                                     */
    int32_t save_adiabaticity;
    int32_t save_start, save_end, save_everystep;
    int32_t block;            /* 0 = automatic                                 */
    tp_term_desc term;
    double budget_s;          /* device wall-clock budget, 0 = default 600 s   */
} tp_hybrid_desc;

int tp_hybrid_run(tp_ctx* ctx, const tp_hybrid_desc* desc, const tp_field* E, const tp_field* B,
                  const double* u0, int64_t n, tp_result** out, tp_result** adia);

/* ---- virtual detectors ----------------------------------------------------
 * get_particle_crossings / get_particle_flux(es) / get_first_crossing of the
 * Meshes extension (ext/TestParticleMeshesExt.jl:98-491), evaluated on the
 * device over packed trajectories: t (total saves), u (total x width, the
 * first 6 values of a row are x, v), nsaved (n; trajectory i owns the next
 * nsaved[i] rows).  A segment between consecutive saves crosses a surface
 * when the signed distances s1, s2 of its end points satisfy s1 s2 < 0 or
 * (s1 != 0 and s2 == 0); the crossing is at f = s1 / (s1 - s2), its state is
 * the linear interpolation of the saves at t = fma(f, t2 - t1, t1); a disk
 * crossing counts only inside the radius.  Pointers may be host or device
 * memory.                                                                    */
enum { TP_SURF_PLANE = 0, TP_SURF_DISK = 1, TP_SURF_SPHERE = 2 };
typedef struct tp_surface {
    int32_t kind;         /* TP_SURF_*                                        */
    int32_t reserved;
    double point[3];      /* PLANE / DISK: point of the plane (the disk's
                             centre); SPHERE: centre                          */
    double normal[3];     /* PLANE / DISK: unit normal                        */
    double radius;        /* DISK / SPHERE                                    */
} tp_surface;
/* Fluxes through disks and spheres: n_flux[j] = sum of weights / area,
 * v_flux[3 j + c] = sum of weight * v_c / area over every crossing of
 * surface j.  weights: n per-trajectory weights, or NULL for `weight`.       */
int tp_detect_fluxes(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                     int64_t n, const tp_surface* surfaces, int32_t nsurf, const double* weights,
                     double weight, double* n_flux, double* v_flux);
/* Crossing velocities and weights per surface: counts[j] crossings of
 * surface j; rows (NULL: count only) receives, surface after surface, one
 * (vx, vy, vz, weight) row per crossing in trajectory and time order.        */
int tp_detect_crossings(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                        int64_t n, const tp_surface* surfaces, int32_t nsurf, const double* weights,
                        double weight, int64_t* counts, double* rows);
/* The interpolated state (6 values) of each trajectory's first crossing of
 * one surface, NaN where it never crosses.                                   */
int tp_detect_first_crossing(tp_ctx* ctx, const double* t, const double* u, int32_t width,
                             const int32_t* nsaved, int64_t n, const tp_surface* surface, double* out);

/* ---- fields and work rates at given states ------------------------------
 * get_fields / get_work (src/boris/boris.jl:599-640): E, B and the work rates
 * of get_work_rates (src/equations.jl:394-441) or get_work_rates_gc
 * (:445-480) at n states, evaluated on the device.                          */
enum {
    TP_POINTS_FULL_ORBIT = 0, /* states (x, v): 6 values                   */
    TP_POINTS_GC = 1          /* states (X, v_par): 4 values                */
};
typedef struct tp_points_desc {
    int32_t kind;        /* TP_POINTS_*                                     */
    int32_t want;        /* bit 0: E and B (6 values); bit 1: the four work
                            rates (P_par, P_fermi, P_grad, P_betatron)     */
    int32_t stride;      /* doubles per state in `u` (>= 6 or >= 4)         */
    int32_t reserved;
    double q2m, m;       /* FULL_ORBIT: charge-to-mass ratio and mass;
                            GC: q2m                                         */
    double q, mu;        /* GC: charge and magnetic moment                  */
} tp_points_desc;
/* u: n states of `stride` doubles; t: n times; out: n rows of
 * 6 * (want & 1) + 4 * ((want >> 1) & 1) doubles.  Host or device memory. */
int tp_eval_points(tp_ctx* ctx, const tp_points_desc* desc, const tp_field* E,
                   const tp_field* B, const double* u, const double* t, int64_t n,
                   double* out);
/* The same with per-point parameters, each optional (NULL: the desc's
 * scalar): q2m_i and m_i (full orbit), q2m_i, q_i and mu_i (guiding
 * centres), n values each, host or device memory.  An ensemble whose
 * particles carry their own q, q/m and mu (the per-particle extension of
 * tp_gc_run) is evaluated in one launch: the reference's get_work /
 * get_fields (boris.jl:594-640) see one p per solve.                      */
int tp_eval_points_params(tp_ctx* ctx, const tp_points_desc* desc,
                          const tp_field* E, const tp_field* B, const double* u,
                          const double* t, const double* q2m_i,
                          const double* m_i, const double* q_i,
                          const double* mu_i, int64_t n, double* out);

/* ---- full-orbit solve (host buffers) --------------------------------------
 * Replaces _solve(::EnsembleAlg, ::TraceProblem, ::AbstractBoris, ...)
 * (src/boris/boris.jl:137-318) and _solve_adaptive (adaptive_boris.jl:40-139)
 * for every trajectory i = 1..N:
 *   u0     6 x N initial states (prob_func already applied on the host, as
 *          src/boris/boris_kernel.jl:290-294 does)
 *   dt_i   optional per-particle dt (fixed step), NULL = desc->dt
 *   tend_i optional per-particle tspan[2], NULL = desc->t1
 * The per-particle arrays are an extension: the reference shares one p, dt
 * and tspan per solve (boris.jl:485).                                       */
int tp_boris_run(tp_ctx* ctx, const tp_run_desc* desc, const tp_field* E,
                 const tp_field* B, const double* u0, const double* dt_i,
                 const double* tend_i, int64_t n, tp_result** out);

/* The same solve from host arrays into host arrays in one call: the results
 * of tp_boris_run followed by tp_result_copy, bit for bit.  One kernel runs
 * the ensemble and counts finished particles per chunk of consecutive
 * indices (up to 32 chunks of at least 32768 particles); the queue schedule
 * hands particles out in index order, so chunks finish while the kernel
 * still runs, and each finished chunk is copied to pinned memory and packed
 * into the caller's buffers by host threads meanwhile.  The context keeps
 * the pinned staging (one chunk, at most 256 MB) between calls.  Where
 * chunks cannot finish early (gridded solves processed in cell order, or
 * work rates completed by a post-pass), host threads first-touch the
 * caller's arrays while the kernel runs and the saves are packed on the
 * device afterwards.
 *   cap_rows        rows t_packed and u_packed can hold (n * slots from
 *                   tp_boris_slots always suffices; fewer fails with
 *                   TP_E_ARG once the saves exceed them)
 *   nsaved, retcode, nsteps   n values each
 *   t_packed, u_packed        packed saves as tp_result_copy writes them
 *   total           rows written;  elapsed_ms  device time of the push
 *                   (may be NULL)
 * Runs whose save count is unknown in advance (adaptive without step_cap)
 * return TP_E_UNSUPPORTED: use tp_boris_run.                                */
int tp_boris_run_host(tp_ctx* ctx, const tp_run_desc* desc, const tp_field* E,
                      const tp_field* B, const double* u0, const double* dt_i,
                      const double* tend_i, int64_t n, int64_t cap_rows,
                      int32_t* nsaved, int8_t* retcode, int64_t* nsteps,
                      double* t_packed, double* u_packed, int64_t* total,
                      double* elapsed_ms);

/* Number of save slots per particle that a run needs (host arrays). */
int tp_boris_slots(const tp_run_desc* desc, const double* dt_i,
                   const double* tend_i, int64_t n, int64_t* nslots);

/* Device-buffer variant: every pointer is device memory, the call is
 * asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream).
 * Outputs are slot-major structure-of-arrays:
 *   t_out[k*n + i], u_out[(k*width + c)*n + i]  (width 6, + 6 with fields,
 *   + 4 with work rates)
 * nsaved[i] save count, retcode[i] TP_RET_*, nsteps[i] steps taken.
 * status (device int32) receives a TP_E_* code from the kernel, or 0.      */
int tp_boris_run_device(tp_ctx* ctx, const tp_run_desc* desc,
                        const tp_field* E, const tp_field* B,
                        const double* u0, const double* dt_i,
                        const double* tend_i, int64_t n, int64_t nslots,
                        double* t_out, double* u_out, int32_t* nsaved,
                        int8_t* retcode, int64_t* nsteps, int32_t* status,
                        void* stream);

/* ---- launch tuning and CUDA graphs ------------------------------------------
 * No reference counterpart (KernelAbstractions picks its workgroup size).
 * tp_autotune times every candidate launch shape -- block sizes 64..256 (384
 * for interleaved E/B grids) with the static and the persistent-queue
 * schedule (only the queue where lifetimes can be uneven: adaptive steps or
 * a termination predicate), and for fixed steps in analytic fields one or
 * two particles per thread -- on a sample of the run (the first
 * min(n, 131072) particles of u0, host memory, for at most max_steps
 * steps), keeps the fastest in the
 * context for runs of the same kernel variant whose descriptor leaves block
 * = 0 / schedule = TP_SCHED_AUTO / particles_per_thread = 0, and reports
 * it.                                                                      */
typedef struct tp_tune_result {
    int32_t block;
    int32_t schedule;      /* TP_SCHED_STATIC or TP_SCHED_QUEUE */
    double ms;             /* device time of the chosen shape on the sample */
    double ms_default;     /* the same sample with the untuned default shape */
    int32_t candidates;
    int32_t particles_per_thread;  /* the chosen particles per thread      */
} tp_tune_result;
int tp_autotune(tp_ctx* ctx, const tp_run_desc* desc, const tp_field* E,
                const tp_field* B, const double* u0, int64_t n,
                int64_t max_steps, tp_tune_result* out);

/* A full-orbit solve with fixed device buffers (the arguments of
 * tp_boris_run_device) captured once into a CUDA graph; tp_graph_launch
 * replays it on a stream.  Buffer contents may change between launches
 * (new initial states); the buffers and fields must outlive the graph.      */
typedef struct tp_graph tp_graph;
int tp_boris_graph_create(tp_ctx* ctx, const tp_run_desc* desc,
                          const tp_field* E, const tp_field* B,
                          const double* u0, const double* dt_i,
                          const double* tend_i, int64_t n, int64_t nslots,
                          double* t_out, double* u_out, int32_t* nsaved,
                          int8_t* retcode, int64_t* nsteps, int32_t* status,
                          tp_graph** out);
int tp_graph_launch(tp_graph* graph, void* stream);
void tp_graph_destroy(tp_graph* graph);

/* ---- guiding-centre solve -------------------------------------------------
 * Replaces _solve(::EnsembleAlg, ::TraceGCProblem, ...) (gc_solver.jl:104-161)
 * with _rk4! (rk4_gc.jl:27-130) or _rk45! (rk45_gc.jl:52-173).
 *   y0  4 x N guiding-centre states (X, v_par)
 *   q_i, q2m_i, mu_i  optional per-particle parameters (extension), NULL =
 *   the shared values of desc
 *   dt_i, tend_i      optional per-particle dt (RK4 step / RK45 initial step)
 *                     and tspan[2] (extension), NULL = desc values.         */
int tp_gc_run(tp_ctx* ctx, const tp_gc_desc* desc, const tp_field* E,
              const tp_field* B, const double* y0, const double* q_i,
              const double* q2m_i, const double* mu_i, const double* dt_i,
              const double* tend_i, int64_t n, tp_result** out);

/* prepare_gc (src/gc/gc.jl:13-84) for N full-orbit states at time t:
 * y0_out (4 x N) = (X, v_par), mu_out (N).  q, m shared by all particles.   */
int tp_gc_prepare(tp_ctx* ctx, const tp_field* E, const tp_field* B,
                  const double* xv, int64_t n, double q, double m, double t,
                  double* y0_out, double* mu_out);

/* gc_to_full (src/gc/gc.jl:106-154) for N guiding-centre states y (4 x N,
 * (X, v_par)) with magnetic moments mu (N) at time t: xv_out (6 x N) is the
 * full-orbit state at gyrophase phase_i[i] (phase when phase_i is null).  q,
 * m shared by all particles; host buffers.  With tp_gc_prepare it is the
 * reference's full_to_gc / gc_to_full pair.                                */
int tp_gc_to_full(tp_ctx* ctx, const tp_field* E, const tp_field* B,
                  const double* y, const double* mu, int64_t n, double q, double m,
                  double phase, const double* phase_i, double t, double* xv_out);

/* ---- results ---------------------------------------------------------------
 * Packed, per-trajectory layout of the reference solutions: trajectory i owns
 * saves offset_i .. offset_i + nsaved_i - 1 with offset_i = sum_{j<i} nsaved_j;
 * t_packed[s] is the save time and u_packed[s*width + c] the state of save s. */
int tp_result_info(const tp_result* res, int64_t* n, int32_t* width,
                   int64_t* total_saved);
int tp_result_copy(const tp_result* res, int32_t* nsaved, int8_t* retcode,
                   int64_t* nsteps, double* t_packed, double* u_packed);
/* device time of the solve, milliseconds (CUDA events around the kernels) */
int tp_result_elapsed_ms(const tp_result* res, double* ms);
void tp_result_destroy(tp_result* res);

/* ---- packing without allocation ---------------------------------------------
 * No counterpart in the reference: an addition of this library for callers
 * that must not let a library allocate device memory (their own memory pool
 * owns every buffer, or allocation is off-limits on their latency path).
 * Packs the slot-major output of tp_boris_run_device into the
 * per-trajectory layout of tp_result_copy, on `stream`, using a static
 * device scratch array instead of cudaMalloc:
 *   t_in[k*n + i], u_in[(k*width + c)*n + i], nsaved[i]  (device, as written)
 *   t_out, u_out  device buffers of at least total saves (n * nslots is safe)
 *   total_out     device int64 receiving the number of packed saves
 * n may not exceed TP_NOALLOC_MAX_TRAJECTORIES (else TP_E_ARG).  Calls share
 * the scratch: calls that overlap on the GPU race.  The first call on a
 * device performs a one-time set-up (it looks up the scratch's device
 * address); make it before any stream capture.  The address is kept for the
 * life of the process: after cudaDeviceReset on that device the library
 * must not be called again in the same process.  Negative nsaved entries
 * count as 0, entries above nslots as nslots, as in tp_boris_run.          */
#define TP_NOALLOC_MAX_TRAJECTORIES 1048576
int tp_pack_results_device_noalloc(tp_ctx* ctx, const double* t_in,
                                   const double* u_in, const int32_t* nsaved,
                                   int64_t n, int64_t nslots, int32_t width,
                                   double* t_out, double* u_out,
                                   int64_t* total_out, void* stream);

/* ---- discrete adjoint of the Boris map ------------------------------------
 * No entry point of the reference: there, gradients of a trajectory come from
 * ForwardDiff through the CPU solver.  The map differentiated is the
 * fixed-step Boris solve of tp_boris_run (boris.jl:445-557) from the initial
 * state to the final save:
 *   v_{-1/2} = U(v_0, x_0, -dt/2);  for k = 0..N-1:
 *   v_{k+1/2} = U(v_{k-1/2}, x_k, dt),  x_{k+1} = x_k + dt v_{k+1/2};
 *   v_N = U(v_{N-1/2}, x_N, dt_final)                     (final save)
 * with U the velocity update of boris.jl:19-45, N = round((t1 - t0)/dt), in
 * the FP32C arithmetic of the push kernels, static fields, no termination.
 * tp_adjoint_forward returns (x_N, v_N) and a tape holding the state every
 * `checkpoint_every` steps; tp_adjoint_backward takes dL/d(x_N, v_N) and
 * recomputes each segment from its checkpoint before running it backwards.
 * Gradients:
 *   grad_u0      dL/du0, N x 6 (float64)
 *   grad_E/B     for grid fields: dL/d(node values), laid out like the
 *                field's data (component fastest), float64; NULL to skip.
 *                They are accumulated in float32 with a power-of-two scale
 *                chosen per pass, so they span float64's range; in a chaotic
 *                field they grow exponentially with the number of steps
 *   grad_param   6 float64: for E then B, dL/dtheta with theta = the dipole
 *                moment for a dipole field, else a uniform offset added to
 *                the field (for a grid: the sum of the node gradients)
 * The fields must outlive the tape and must not be updated in between.     */
typedef struct tp_adj_desc {
    tp_run_desc run;           /* alg TP_ALG_BORIS, precision TP_PREC_FP32C,
                                  term.flags 0; t0, t1, dt, q2m, block     */
    int64_t checkpoint_every;  /* K >= 1 steps per checkpoint segment, or
                                  0: automatic (2 for an interleaved E/B
                                  grid when the tape fits in half of the
                                  free device memory, else 64).  The tape
                                  holds 48 bytes per particle per segment;
                                  E/B-grid segments of <= 8 steps run the
                                  one-kernel backward, longer ones two
                                  kernels per segment                     */
} tp_adj_desc;

typedef struct tp_tape tp_tape;

/* host buffers: u0 and u_final N x 6 */
int tp_adjoint_forward(tp_ctx* ctx, const tp_adj_desc* desc, const tp_field* E,
                       const tp_field* B, const double* u0, int64_t n,
                       double* u_final, tp_tape** tape);
int tp_adjoint_backward(tp_tape* tape, const double* grad_final,
                        double* grad_u0, double* grad_E, double* grad_B,
                        double* grad_param);
/* device buffers, on `stream` (a cudaStream_t); the backward pass waits for
 * its stream once, to check the range of the node gradients (see above)    */
int tp_adjoint_forward_device(tp_ctx* ctx, const tp_adj_desc* desc,
                              const tp_field* E, const tp_field* B,
                              const double* u0, int64_t n, double* u_final,
                              tp_tape** tape, void* stream);
int tp_adjoint_backward_device(tp_tape* tape, const double* grad_final,
                               double* grad_u0, double* grad_E, double* grad_B,
                               double* grad_param, void* stream);
/* Re-record an existing tape for new initial states (same N), reusing its
 * device memory; fields updated with tp_field_update since are picked up.
 * For optimisation loops: rerun, then backward, without reallocation.     */
int tp_tape_rerun_device(tp_tape* tape, const double* u0, double* u_final,
                         void* stream);
/* device bytes a tape holds (checkpoints, and after the first backward pass
 * the segment records and gradient tables), and its step count N */
int tp_tape_info(const tp_tape* tape, int64_t* device_bytes, int64_t* nsteps);
/* Steps per checkpoint segment the tape uses (the automatic choice resolved)
 * and the number of segments; either pointer may be null. */
int tp_tape_segments(const tp_tape* tape, int64_t* checkpoint_every, int64_t* segments);
void tp_tape_destroy(tp_tape* tape);

#ifdef __cplusplus
}
#endif

#endif /* TP_ABI_H */
