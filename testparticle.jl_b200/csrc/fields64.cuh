// fields64.cuh -- float64 field evaluation and Boris / Multistep velocity
// updates.  Included only by translation units compiled with -fmad=false:
// the expressions follow the reference's operation order without contraction,
// and the places where the reference fuses (@muladd on scalars) call fma()
// explicitly, so results equal the CPU restatement bit for bit wherever only
// +, -, *, /, sqrt and fma are involved.
#pragma once

#include "grid_general.cuh"
#include "ptrig.cuh"
#include "tp_device.cuh"

namespace tpb {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ double abs2sum(D3 a) { return (a.x * a.x + a.y * a.y) + a.z * a.z; }
__device__ __forceinline__ double norm(D3 a) { return sqrt(abs2sum(a)); }

// ---------------------------------------------------------------- grid axis
// Per-axis cell index and fraction of the trilinear interpolant (the
// FieldInterpolator of src/utility/interpolation.jl:217-235, boundary rules
// FillExtrap(NaN) / ClampExtrap() / PeriodicBC(endpoint=:exclusive)).
struct Ax {
    int32_t i0, i1;
    double f;
};

__device__ __forceinline__ bool grid_axis(const DevField& g, int a, double x, Ax& o) {
    double u = (x - g.x0[a]) * g.inv_dx[a];
    int32_t na = g.n[a];
    if (g.bc == TP_BC_PERIODIC) {
        double fl = floor(u);
        o.f = u - fl;
        long long i = (long long)fl % (long long)na;
        if (i < 0) i += na;
        o.i0 = (int32_t)i;
        o.i1 = (o.i0 + 1 == na) ? 0 : o.i0 + 1;
        return true;
    }
    double umax = (double)(na - 1);
    if (g.bc == TP_BC_CLAMP) {
        u = (u < 0.0) ? 0.0 : u;
        u = (umax < u) ? umax : u;
    } else if (!(u >= 0.0 && u <= umax)) {
        return false;
    }
    double fl = floor(u);
    long long i = (long long)fl;
    if (i > na - 2) i = na - 2;
    o.i0 = (int32_t)i;
    o.i1 = o.i0 + 1;
    o.f = u - (double)i;
    return true;
}

__device__ __forceinline__ double lerp64(double a, double b, double f) { return a + f * (b - a); }

// Load node `node` of a table with `stride` 4-vectors per node, at offset `off`.
__device__ __forceinline__ D3 load_node(const void* tab, bool f64, int64_t idx) {
    if (f64) {
        const double2* p = reinterpret_cast<const double2*>(tab) + 2 * idx;
        double2 a = __ldg(p), b = __ldg(p + 1);
        return {a.x, a.y, b.x};
    }
    float4 q = __ldg(reinterpret_cast<const float4*>(tab) + idx);
    return {(double)q.x, (double)q.y, (double)q.z};
}

// Trilinear interpolation from precomputed axes; `stride`/`off` select a
// field inside an interleaved table (stride 2: E at off 0, B at off 1).
__device__ __forceinline__ D3 tri64(const DevField& g, const void* tab, bool f64, int stride,
                                    int off, const Ax& ax, const Ax& ay, const Ax& az) {
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    int64_t j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
    D3 v000 = load_node(tab, f64, (ax.i0 + j0 + k0) * stride + off);
    D3 v100 = load_node(tab, f64, (ax.i1 + j0 + k0) * stride + off);
    D3 v010 = load_node(tab, f64, (ax.i0 + j1 + k0) * stride + off);
    D3 v110 = load_node(tab, f64, (ax.i1 + j1 + k0) * stride + off);
    D3 v001 = load_node(tab, f64, (ax.i0 + j0 + k1) * stride + off);
    D3 v101 = load_node(tab, f64, (ax.i1 + j0 + k1) * stride + off);
    D3 v011 = load_node(tab, f64, (ax.i0 + j1 + k1) * stride + off);
    D3 v111 = load_node(tab, f64, (ax.i1 + j1 + k1) * stride + off);
    D3 o;
#define TPB_TRI(c)                                              \
    {                                                           \
        double c00 = lerp64(v000.c, v100.c, ax.f);              \
        double c10 = lerp64(v010.c, v110.c, ax.f);              \
        double c01 = lerp64(v001.c, v101.c, ax.f);              \
        double c11 = lerp64(v011.c, v111.c, ax.f);              \
        double c0 = lerp64(c00, c10, ay.f);                     \
        double c1 = lerp64(c01, c11, ay.f);                     \
        o.c = lerp64(c0, c1, az.f);                             \
    }
    TPB_TRI(x)
    TPB_TRI(y)
    TPB_TRI(z)
#undef TPB_TRI
    return o;
}

__device__ __forceinline__ D3 nan3() {
    double q = __longlong_as_double(0x7ff8000000000000ULL);
    return {q, q, q};
}

__device__ __forceinline__ bool grid_axes64(const DevField& g, D3 r, Ax& ax, Ax& ay, Ax& az) {
    bool ok = grid_axis(g, 0, r.x, ax);
    ok = grid_axis(g, 1, r.y, ay) && ok;
    ok = grid_axis(g, 2, r.z, az) && ok;
    return ok;
}

// grids off the fast path (grid_general.cuh): value, and value with Jacobian
static __device__ __noinline__ D3 grid_general64(const DevField& g, D3 r) {
    double p[3] = {r.x, r.y, r.z}, o[3];
    if (!grid_general_eval<double>(g, p, o)) return nan3();
    return {o[0], o[1], o[2]};
}

static __device__ __noinline__ void grid_general_jac64(const DevField& g, D3 r, D3& F, double J[9]) {
    Dual3 p[3] = {{r.x, {1.0, 0.0, 0.0}}, {r.y, {0.0, 1.0, 0.0}}, {r.z, {0.0, 0.0, 1.0}}}, o[3];
    if (!grid_general_eval<Dual3>(g, p, o)) {
        F = nan3();
        for (int k = 0; k < 9; ++k) J[k] = F.x;
        return;
    }
    F = {o[0].v, o[1].v, o[2].v};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[3 * i + j] = o[i].d[j];
}

// GEN = false: the caller guarantees no general grid reaches it (kernels
// specialised for trilinear grids keep the general code out of their body)
template <bool GEN = true>
__device__ __forceinline__ D3 grid_eval64(const DevField& g, D3 r) {
    if (GEN && g.general) return grid_general64(*g.self, r);
    Ax ax, ay, az;
    if (!grid_axes64(g, r, ax, ay, az)) return nan3();
    return tri64(g, g.tab, g.f64 != 0, 1, 0, ax, ay, az);
}

// Analytic fields: ZERO, UNIFORM, AFFINE, DIPOLE (order of the oracle).
__device__ __forceinline__ D3 analytic_eval64(const DevField& f, D3 r, double t) {
    switch (f.kind) {
        case TP_FIELD_UNIFORM:
            return {f.v[0], f.v[1], f.v[2]};
        case TP_FIELD_AFFINE: {
            D3 o;
            o.x = (f.v[0] + ((f.J[0] * r.x + f.J[1] * r.y) + f.J[2] * r.z)) + f.rate[0] * t;
            o.y = (f.v[1] + ((f.J[3] * r.x + f.J[4] * r.y) + f.J[5] * r.z)) + f.rate[1] * t;
            o.z = (f.v[2] + ((f.J[6] * r.x + f.J[7] * r.y) + f.J[8] * r.z)) + f.rate[2] * t;
            return o;
        }
        case TP_FIELD_DIPOLE: {
            D3 d = r - D3{f.c[0], f.c[1], f.c[2]};
            D3 m{f.m[0], f.m[1], f.m[2]};
            double dm = norm(d);
            D3 rh = d / dm;
            double mr = dot(m, rh);
            double d3 = (dm * dm) * dm;
            D3 s = (3.0 * mr) * rh - m;
            return (f.coef * s) / d3;
        }
        default:
            return {0.0, 0.0, 0.0};
    }
}

__device__ __forceinline__ D3 quad_eval64(const DevField& f, D3 r, double t) {
    double o[3];
    quad_eval(f, r.x, r.y, r.z, t, o);
    return {o[0], o[1], o[2]};
}

// ---------------------------------------------------------------- time series
// LazyTimeInterpolator (src/utility/interpolation.jl:337-430): k = the
// number of snapshot times <= t (searchsortedlast); k == 0 or k == n clamp
// to the first / last snapshot, otherwise w = (t - t_k) / (t_{k+1} - t_k)
// and the value is (1 - w) F_k + w F_{k+1}.  Snapshots are never series.
__device__ __forceinline__ D3 snapshot_eval64(const DevField& f, D3 r, double t) {
    if (f.kind == TP_FIELD_GRID) return grid_eval64<true>(f, r);
    if (f.kind == TP_FIELD_QUADRATIC) return quad_eval64(f, r, t);
    return analytic_eval64(f, r, t);
}

__device__ __forceinline__ int series_index(const DevField& f, double t) {
    int lo = 0, hi = f.nts;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(f.ts + mid) <= t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static __device__ __noinline__ D3 series_eval64(const DevField& f, D3 r, double t) {
    const int k = series_index(f, t);
    if (k == 0) return snapshot_eval64(f.snaps[0], r, t);
    if (k >= f.nts) return snapshot_eval64(f.snaps[f.nts - 1], r, t);
    const double t1 = __ldg(f.ts + k - 1), t2 = __ldg(f.ts + k);
    const double w = (t - t1) / (t2 - t1);
    D3 a = snapshot_eval64(f.snaps[k - 1], r, t), b = snapshot_eval64(f.snaps[k], r, t);
    return (1.0 - w) * a + w * b;
}

// derivative_t: (F_{k+1} - F_k) / (t_{k+1} - t_k) inside, zero outside
static __device__ __noinline__ D3 series_dtime64(const DevField& f, D3 r, double t) {
    const int k = series_index(f, t);
    if (k == 0 || k >= f.nts) return {0.0, 0.0, 0.0};
    const double t1 = __ldg(f.ts + k - 1), t2 = __ldg(f.ts + k);
    D3 a = snapshot_eval64(f.snaps[k - 1], r, t), b = snapshot_eval64(f.snaps[k], r, t);
    return (b - a) / (t2 - t1);
}

template <bool GEN = true>
__device__ __forceinline__ D3 field_eval64(const DevField& f, D3 r, double t) {
    if (f.kind == TP_FIELD_GRID) return grid_eval64<GEN>(f, r);
    if (f.kind == TP_FIELD_QUADRATIC) return quad_eval64(f, r, t);
    if (GEN && f.kind == TP_FIELD_SERIES) return series_eval64(*f.self, r, t);
    return analytic_eval64(f, r, t);
}

// E and B at one point (one gather pass when the two grids are interleaved).
__device__ __forceinline__ void eval_EB64(const DevFields& F, D3 r, double t, D3& E, D3& B) {
    if (F.eb) {
        // both grids on one geometry: one axis computation, one gather pass
        Ax ax, ay, az;
        if (!grid_axes64(F.B, r, ax, ay, az)) {
            E = nan3();
            B = E;
            return;
        }
        bool f64 = F.eb_f64 != 0;
        E = tri64(F.B, F.eb, f64, 2, 0, ax, ay, az);
        B = tri64(F.B, F.eb, f64, 2, 1, ax, ay, az);
        return;
    }
    E = field_eval64(F.E, r, t);
    B = field_eval64(F.B, r, t);
}

// One 32-byte node record (E xyz0, B xyz0) of the float interleaved table in
// a single 256-bit read-only load (sm_100 ld.global.nc.v8).
__device__ __forceinline__ void ldg_node8_64(const float4* p, float4& e, float4& b) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(e.x), "=f"(e.y), "=f"(e.z), "=f"(e.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// E and B from the float interleaved table, interpolated in float64 in the
// order of tri64 (the values are exact float -> double conversions)
__device__ __forceinline__ void eb_eval64_f32(const DevFields& F, D3 r, D3& E, D3& B) {
    Ax ax, ay, az;
    if (!grid_axes64(F.B, r, ax, ay, az)) {
        E = nan3();
        B = E;
        return;
    }
    const float4* T = F.eb32;
    const int64_t nx = F.B.n[0], nxy = (int64_t)F.B.n[0] * F.B.n[1];
    int64_t j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
    float4 e000, b000, e100, b100, e010, b010, e110, b110;
    float4 e001, b001, e101, b101, e011, b011, e111, b111;
    ldg_node8_64(T + 2 * (ax.i0 + j0 + k0), e000, b000);
    ldg_node8_64(T + 2 * (ax.i1 + j0 + k0), e100, b100);
    ldg_node8_64(T + 2 * (ax.i0 + j1 + k0), e010, b010);
    ldg_node8_64(T + 2 * (ax.i1 + j1 + k0), e110, b110);
    ldg_node8_64(T + 2 * (ax.i0 + j0 + k1), e001, b001);
    ldg_node8_64(T + 2 * (ax.i1 + j0 + k1), e101, b101);
    ldg_node8_64(T + 2 * (ax.i0 + j1 + k1), e011, b011);
    ldg_node8_64(T + 2 * (ax.i1 + j1 + k1), e111, b111);
#define TPB_TRI64F(dst, q, c)                                                                  \
    {                                                                                          \
        double c00 = lerp64((double)(q##000).c, (double)(q##100).c, ax.f);                         \
        double c10 = lerp64((double)(q##010).c, (double)(q##110).c, ax.f);                         \
        double c01 = lerp64((double)(q##001).c, (double)(q##101).c, ax.f);                         \
        double c11 = lerp64((double)(q##011).c, (double)(q##111).c, ax.f);                         \
        double c0 = lerp64(c00, c10, ay.f);                                                    \
        double c1 = lerp64(c01, c11, ay.f);                                                    \
        dst.c = lerp64(c0, c1, az.f);                                                          \
    }
    TPB_TRI64F(E, e, x)
    TPB_TRI64F(E, e, y)
    TPB_TRI64F(E, e, z)
    TPB_TRI64F(B, b, x)
    TPB_TRI64F(B, b, y)
    TPB_TRI64F(B, b, z)
#undef TPB_TRI64F
}

template <int FK>
__device__ __forceinline__ void eval_EB64t(const DevFields& F, D3 r, double t, D3& E, D3& B) {
    if (FK == FK_ANALYTIC) {
        E = analytic_eval64(F.E, r, t);
        B = analytic_eval64(F.B, r, t);
    } else if (FK == FK_EBGRID) {
        eb_eval64_f32(F, r, E, B);
    } else {
        E = field_eval64<FK == FK_GENGRID>(F.E, r, t);
        B = field_eval64<FK == FK_GENGRID>(F.B, r, t);
    }
}

__device__ __forceinline__ bool fields_static(const DevFields& F) {
    bool e = !((F.E.kind == TP_FIELD_AFFINE || F.E.kind == TP_FIELD_QUADRATIC) &&
               (F.E.rate[0] != 0.0 || F.E.rate[1] != 0.0 || F.E.rate[2] != 0.0));
    bool b = !((F.B.kind == TP_FIELD_AFFINE || F.B.kind == TP_FIELD_QUADRATIC) &&
               (F.B.rate[0] != 0.0 || F.B.rate[1] != 0.0 || F.B.rate[2] != 0.0));
    return e && b && F.E.kind != TP_FIELD_SERIES && F.B.kind != TP_FIELD_SERIES;
}

// ---------------------------------------------------------------- updates
// boris_velocity_update, src/boris/boris.jl:19-31, with qdt_2m = q2m*0.5*dt
// (update_velocity, boris.jl:38-45)
__device__ __forceinline__ D3 boris_rot64(D3 v, D3 E, D3 B, double q2m, double dt) {
    double qdt_2m = q2m * 0.5 * dt;
    D3 t_rotate = qdt_2m * B;
    double t_mag2 = abs2sum(t_rotate);
    D3 s_rotate = (2.0 * t_rotate) / (1.0 + t_mag2);
    D3 vm = v + qdt_2m * E;
    D3 vp_ = vm + cross(vm, t_rotate);
    D3 vplus = vm + cross(vp_, s_rotate);
    return vplus + qdt_2m * E;
}

// update_velocity_multistep, src/boris/multistep_boris.jl:65-142
__device__ __forceinline__ D3 multistep_rot64(D3 v, D3 E, D3 B, double q2m, double dt, int N,
                                              int n) {
    double factor = q2m * dt / (double)(2 * n);
    D3 t_n = factor * B;
    D3 e_n = factor * E;
    if (N != 2) {
        double t_mag2 = abs2sum(t_n);
        double f_N, e_corr;
        if (N == 4) {
            f_N = 1.0 + t_mag2 / 3.0;
            e_corr = -1.0 / 3.0;
        } else {
            f_N = (1.0 + t_mag2 / 3.0) + 2.0 * t_mag2 * t_mag2 / 15.0;
            e_corr = -1.0 / 3.0 - 2.0 * t_mag2 / 15.0;
        }
        double e_dot_t = dot(e_n, t_n);
        e_n = f_N * e_n + (e_corr * e_dot_t) * t_n;
        t_n = f_N * t_n;
    }
    double t_n_mag2 = abs2sum(t_n);
    double t_n_mag = sqrt(t_n_mag2);
    double c1, c2, c3, c6;
    double nd = (double)n;
    if (t_n_mag < 1.0e-4) {
        c1 = fma(-(2.0 * nd * nd), t_n_mag2, 1.0);
        double n_term1 = 2.0 * nd;
        double n_term3 = 4.0 * nd * nd * nd;
        c2 = fma(-((n_term1 + n_term3) / 3.0), t_n_mag2, n_term1);
        c3 = fma(-((4.0 * nd * nd + 2.0 * nd * nd * nd * nd) / 3.0), t_n_mag2, 2.0 * nd * nd);
        c6 = (n_term1 + n_term3) / 3.0;
    } else {
        // atan and sincos of the reference, as the portable routines the
        // oracle shares (ptrig.cuh): the same bits on the device and the CPU
        double alpha = patan2(t_n_mag, 1.0);
        double s, c;
        psincos(nd * alpha, s, c);
        double s2 = 2.0 * s * c;
        c1 = fma(c, c, -(s * s));
        c2 = s2 / t_n_mag;
        c3 = 2.0 * s * s / t_n_mag2;
        c6 = (2.0 * nd - c2) / t_n_mag2;
    }
    double v_dot_t = dot(v, t_n);
    double e_dot_t = dot(e_n, t_n);
    D3 v_cross_t = cross(v, t_n);
    D3 e_cross_t = cross(e_n, t_n);
    D3 out = c1 * v + c2 * v_cross_t;
    out = out + (c3 * v_dot_t) * t_n;
    out = out + c2 * e_n;
    out = out + c3 * e_cross_t;
    out = out + (c6 * e_dot_t) * t_n;
    return out;
}

template <bool MULTI>
__device__ __forceinline__ D3 vel_update64(D3 v, D3 E, D3 B, double q2m, double dt, int N, int n) {
    if (MULTI) return multistep_rot64(v, E, B, q2m, dt, N, n);
    return boris_rot64(v, E, B, q2m, dt);
}

// isoutside(u, p, t) restated for the flag predicates of tp_term_desc
__device__ __forceinline__ bool outside64(const DevTerm& T, D3 r, D3 v, double t) {
    int f = T.flags;
    if (f & TP_TERM_NAN)
        if (isnan(r.x) || isnan(r.y) || isnan(r.z) || isnan(v.x) || isnan(v.y) || isnan(v.z))
            return true;
    if (f & TP_TERM_SHELL) {
        double rr = sqrt((r.x * r.x + r.y * r.y) + r.z * r.z);
        if (rr < T.rmin || rr > T.rmax) return true;
    }
    if (f & TP_TERM_BOX) {
        if (r.x < T.lo[0] || r.x > T.hi[0]) return true;
        if (r.y < T.lo[1] || r.y > T.hi[1]) return true;
        if (r.z < T.lo[2] || r.z > T.hi[2]) return true;
    }
    if (f & TP_TERM_TIME)
        if (t > T.tmax) return true;
    return false;
}

// B and its Jacobian (row-major J[i][j] = dB_i/dx_j), float64, in the order
// of the CPU restatement (the role of ForwardDiff in _get_B_jacobian,
// src/utility/utility.jl:386-392)
// Field configurations of the float64 Jacobian and value helpers: GM_ANALYTIC
// (no grids), GM_GRID (trilinear uniform Cartesian grids only), GM_ANY (also
// the general grids of grid_general.cuh).
enum { GM_ANALYTIC = 0, GM_GRID = 1, GM_ANY = 2, GM_LEAF = 3 };  // GM_LEAF: GM_ANY but no series

// the grid mode of a full-orbit kernel's field configuration
template <int FK>
struct GMOf {
    static constexpr int value = FK == FK_ANALYTIC ? GM_ANALYTIC : (FK == FK_GENGRID ? GM_ANY : GM_GRID);
};

static __device__ __noinline__ void series_jac64(const DevField& f, D3 r, double t, D3& F, double J[9]);

template <int GM>
__device__ __forceinline__ void field_jac64(const DevField& f, D3 r, double t, D3& F, double J[9]) {
    constexpr bool GRID = GM != GM_ANALYTIC;
    for (int k = 0; k < 9; ++k) J[k] = 0.0;
    switch (f.kind) {
        case TP_FIELD_UNIFORM:
            F = {f.v[0], f.v[1], f.v[2]};
            return;
        case TP_FIELD_AFFINE:
            F = analytic_eval64(f, r, t);
            for (int k = 0; k < 9; ++k) J[k] = f.J[k];
            return;
        case TP_FIELD_QUADRATIC: {
            if (!GRID) {  // never selected: quadratic fields take the generic kernels
                F = {0.0, 0.0, 0.0};
                return;
            }
            F = quad_eval64(f, r, t);
            // dF_i/dx_j = J_ij + sum_k (Q_ijk + Q_ikj) x_k
            const double x[3] = {r.x, r.y, r.z};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double* Q = f.Q + 9 * i;
                    double acc = f.J[3 * i + j];
                    for (int k = 0; k < 3; ++k) acc = acc + (Q[3 * j + k] + Q[3 * k + j]) * x[k];
                    J[3 * i + j] = acc;
                }
            return;
        }
        case TP_FIELD_DIPOLE: {
            F = analytic_eval64(f, r, t);
            D3 d = r - D3{f.c[0], f.c[1], f.c[2]};
            double d2 = abs2sum(d);
            double dm = sqrt(d2);
            double inv5 = 1.0 / ((d2 * d2) * dm);
            double inv7 = inv5 / d2;
            double md = dot(D3{f.m[0], f.m[1], f.m[2]}, d);
            double dv[3] = {d.x, d.y, d.z};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double dij = (i == j) ? md : 0.0;
                    J[3 * i + j] = f.coef * (3.0 * ((f.m[j] * dv[i] + dij) + f.m[i] * dv[j]) * inv5 -
                                             15.0 * md * dv[i] * dv[j] * inv7);
                }
            return;
        }
        case TP_FIELD_GRID: {
            if (!GRID) {
                F = {0.0, 0.0, 0.0};
                return;
            }
            if ((GM == GM_ANY || GM == GM_LEAF) && f.general) {
                grid_general_jac64(*f.self, r, F, J);
                return;
            }
            Ax ax, ay, az;
            if (!grid_axes64(f, r, ax, ay, az)) {
                F = nan3();
                for (int k = 0; k < 9; ++k) J[k] = F.x;
                return;
            }
            F = tri64(f, f.tab, f.f64 != 0, 1, 0, ax, ay, az);
            double sx = f.inv_dx[0], sy = f.inv_dx[1], sz = f.inv_dx[2];
            if (f.bc == TP_BC_CLAMP) {
                double ux = (r.x - f.x0[0]) * f.inv_dx[0], uy = (r.y - f.x0[1]) * f.inv_dx[1],
                       uz = (r.z - f.x0[2]) * f.inv_dx[2];
                if (ux < 0.0 || ux > (double)(f.n[0] - 1)) sx = 0.0;
                if (uy < 0.0 || uy > (double)(f.n[1] - 1)) sy = 0.0;
                if (uz < 0.0 || uz > (double)(f.n[2] - 1)) sz = 0.0;
            }
            const int64_t nx = f.n[0], nxy = (int64_t)f.n[0] * f.n[1];
            int64_t j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
            bool f64 = f.f64 != 0;
            D3 w000 = load_node(f.tab, f64, ax.i0 + j0 + k0), w100 = load_node(f.tab, f64, ax.i1 + j0 + k0);
            D3 w010 = load_node(f.tab, f64, ax.i0 + j1 + k0), w110 = load_node(f.tab, f64, ax.i1 + j1 + k0);
            D3 w001 = load_node(f.tab, f64, ax.i0 + j0 + k1), w101 = load_node(f.tab, f64, ax.i1 + j0 + k1);
            D3 w011 = load_node(f.tab, f64, ax.i0 + j1 + k1), w111 = load_node(f.tab, f64, ax.i1 + j1 + k1);
            double fx = ax.f, fy = ay.f, fz = az.f;
#define TPB_GJ(c, row)                                                                  \
    {                                                                                   \
        double v000 = w000.c, v100 = w100.c, v010 = w010.c, v110 = w110.c;              \
        double v001 = w001.c, v101 = w101.c, v011 = w011.c, v111 = w111.c;              \
        double dx00 = v100 - v000, dx10 = v110 - v010, dx01 = v101 - v001, dx11 = v111 - v011; \
        double dx0 = lerp64(dx00, dx10, fy), dx1 = lerp64(dx01, dx11, fy);              \
        J[3 * row + 0] = lerp64(dx0, dx1, fz) * sx;                                     \
        double c00 = lerp64(v000, v100, fx), c10 = lerp64(v010, v110, fx);              \
        double c01 = lerp64(v001, v101, fx), c11 = lerp64(v011, v111, fx);              \
        J[3 * row + 1] = lerp64(c10 - c00, c11 - c01, fz) * sy;                         \
        double c0 = lerp64(c00, c10, fy), c1 = lerp64(c01, c11, fy);                    \
        J[3 * row + 2] = (c1 - c0) * sz;                                                \
    }
            TPB_GJ(x, 0)
            TPB_GJ(y, 1)
            TPB_GJ(z, 2)
#undef TPB_GJ
            return;
        }
        case TP_FIELD_SERIES:
            if (GM == GM_ANY) {
                series_jac64(*f.self, r, t, F, J);
                return;
            }
            F = {0.0, 0.0, 0.0};
            return;
        default:
            F = {0.0, 0.0, 0.0};
            return;
    }
}

// Jacobian of a series: (1 - w) J_k + w J_{k+1} (clamped outside)
static __device__ __noinline__ void series_jac64(const DevField& f, D3 r, double t, D3& F, double J[9]) {
    const int k = series_index(f, t);
    if (k == 0 || k >= f.nts) {
        field_jac64<GM_LEAF>(f.snaps[k == 0 ? 0 : f.nts - 1], r, t, F, J);
        return;
    }
    const double t1 = __ldg(f.ts + k - 1), t2 = __ldg(f.ts + k);
    const double w = (t - t1) / (t2 - t1);
    D3 Fa, Fb;
    double Ja[9], Jb[9];
    field_jac64<GM_LEAF>(f.snaps[k - 1], r, t, Fa, Ja);
    field_jac64<GM_LEAF>(f.snaps[k], r, t, Fb, Jb);
    F = (1.0 - w) * Fa + w * Fb;
    for (int q = 0; q < 9; ++q) J[q] = (1.0 - w) * Ja[q] + w * Jb[q];
}

template <int GM>
__device__ __forceinline__ D3 field_val64(const DevField& f, D3 r, double t) {
    if (GM != GM_ANALYTIC) return field_eval64<GM == GM_ANY || GM == GM_LEAF>(f, r, t);
    return analytic_eval64(f, r, t);
}

// get_magnetic_properties (src/utility/utility.jl:409-422) with
// _get_curvature (:379-384): B, grad|B| = JB^T b, curvature
// kappa = (JB b - b (grad|B| . b)) / |B|, b = B / |B|
struct MagProps {
    D3 B, gradB, kappa, bh;
    double Bmag;
};

template <int GM>
__device__ __forceinline__ MagProps magnetic_properties64(const DevField& f, D3 r, double t) {
    MagProps m;
    double J[9];
    field_jac64<GM>(f, r, t, m.B, J);
    m.Bmag = norm(m.B);
    if (m.Bmag == 0.0) {
        m.gradB = m.kappa = m.bh = D3{0.0, 0.0, 0.0};
        return m;
    }
    const D3 b = m.B / m.Bmag;
    m.bh = b;
    m.gradB = {(J[0] * b.x + J[3] * b.y) + J[6] * b.z, (J[1] * b.x + J[4] * b.y) + J[7] * b.z,
               (J[2] * b.x + J[5] * b.y) + J[8] * b.z};
    const D3 Jb{(J[0] * b.x + J[1] * b.y) + J[2] * b.z, (J[3] * b.x + J[4] * b.y) + J[5] * b.z,
                (J[6] * b.x + J[7] * b.y) + J[8] * b.z};
    m.kappa = (Jb + b * (-dot(m.gradB, b))) / m.Bmag;
    return m;
}

// dB/dt of a field: the rate of a time-dependent affine field, else 0
// (derivative_t, src/prepare.jl:64-74)
template <int GM>
__device__ __forceinline__ D3 field_dtime64(const DevField& f, D3 r, double t) {
    if (f.kind == TP_FIELD_AFFINE || f.kind == TP_FIELD_QUADRATIC) return {f.rate[0], f.rate[1], f.rate[2]};
    if (GM == GM_ANY && f.kind == TP_FIELD_SERIES) return series_dtime64(*f.self, r, t);
    return {0.0, 0.0, 0.0};
}

// The four work rates of a saved state (P_par, P_fermi, P_grad, P_betatron)
// from E, the magnetic properties, v_par and mu (get_work_rates,
// src/equations.jl:394-441; get_work_rates_gc, :445-480)
__device__ __forceinline__ void work_terms64(const MagProps& mp, D3 E, D3 dBdt, double q, double m, double vpar,
                                             double mu, double* W) {
    W[0] = q * vpar * dot(E, mp.bh);
    W[1] = (m * (vpar * vpar) / mp.Bmag) * dot(cross(mp.bh, mp.kappa), E);
    W[2] = (mu / mp.Bmag) * dot(cross(mp.bh, mp.gradB), E);
    W[3] = mu * dot(dBdt, mp.bh);
}

// full orbit: v_par = v . b, mu = m |v - v_par b|^2 / (2 |B|), q = q2m m
template <int GM>
__device__ __forceinline__ void work_rates64(const DevFields& F, D3 r, D3 v, double t, double q2m, double m,
                                             double* W) {
    const double q = q2m * m;
    const D3 E = field_val64<GM>(F.E, r, t);
    const MagProps mp = magnetic_properties64<GM>(F.B, r, t);
    if (mp.Bmag == 0.0) {
        W[0] = W[1] = W[2] = W[3] = 0.0;
        return;
    }
    const double vpar = dot(v, mp.bh);
    const D3 vperp = v - vpar * mp.bh;
    const double mu = m * dot(vperp, vperp) / (2.0 * mp.Bmag);
    work_terms64(mp, E, field_dtime64<GM>(F.B, r, t), q, m, vpar, mu, W);
}

// guiding centre: state (X, v_par), mu given, m = q / q2m
template <int GM>
__device__ __forceinline__ void work_rates_gc64(const DevFields& F, D3 X, double vpar, double t, double q,
                                                double q2m, double mu, double* W) {
    const D3 E = field_val64<GM>(F.E, X, t);
    const MagProps mp = magnetic_properties64<GM>(F.B, X, t);
    if (mp.Bmag == 0.0) {
        W[0] = W[1] = W[2] = W[3] = 0.0;
        return;
    }
    work_terms64(mp, E, field_dtime64<GM>(F.B, X, t), q, q / q2m, vpar, mu, W);
}

}  // namespace tpb
