// fp32c_common.cuh -- float32 compensated-position arithmetic shared by the
// FP32C push kernels (boris_fp32c.cu) and the discrete adjoint (adjoint.cu):
// compensated positions and velocities, the float cell index, trilinear
// gathers from the interleaved E/B table, analytic fields, and the Boris and
// Multistep velocity updates in delta form.
#pragma once

#include "fields64.cuh"
#include "grid_general.cuh"
#include "tp_device.cuh"

namespace tpb {

namespace {

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Compensated position: x = hi + lo + w * L (w only on wrapped axes)
struct CPos {
    float hi[3], lo[3];
    int w[3];
};

// TwoSum (Knuth) + Fast2Sum (Dekker): (hi, lo) += d
__device__ __forceinline__ void cadd(float& hi, float& lo, float d) {
    float s = __fadd_rn(hi, d);
    float bb = __fsub_rn(s, hi);
    float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(d, bb));
    e = __fadd_rn(e, lo);
    float h = __fadd_rn(s, e);
    lo = __fsub_rn(e, __fsub_rn(h, s));
    hi = h;
}

__device__ __forceinline__ double cpos_value(const BorisArgs& a, const CPos& p, int c) {
    double x = (double)p.hi[c] + (double)p.lo[c];
    if (a.wrap[c]) x += (double)p.w[c] * a.wrapL[c];
    return x;
}

__device__ __forceinline__ void cpos_init(const BorisArgs& a, CPos& p, const double* x) {
    for (int c = 0; c < 3; ++c) {
        double v = x[c];
        p.w[c] = 0;
        if (a.wrap[c]) {
            double k = floor((v - a.wrap0[c]) / a.wrapL[c]);
            p.w[c] = (int)k;
            v = v - k * a.wrapL[c];
        }
        p.hi[c] = (float)v;
        p.lo[c] = (float)(v - (double)p.hi[c]);
    }
}

// WRAP = false: the caller knows no axis wraps (analytic fields never do)
template <bool WRAP = true>
__device__ __forceinline__ void cpos_push(const BorisArgs& a, CPos& p, F3 v, float dt) {
    float d[3] = {v.x * dt, v.y * dt, v.z * dt};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        cadd(p.hi[c], p.lo[c], d[c]);
        if (WRAP && a.wrap[c]) {
            float x0 = (float)a.wrap0[c];
            float L = (float)a.wrapL[c];
            if (p.hi[c] >= x0 + L) {
                cadd(p.hi[c], p.lo[c], -L);
                p.w[c] += 1;
            } else if (p.hi[c] < x0) {
                cadd(p.hi[c], p.lo[c], L);
                p.w[c] -= 1;
            }
        }
    }
}

// ---------------------------------------------------------------- fields
struct AxF {
    int i0, i1;
    float f;
    float ds;  // d f / d x: 1/dx, or 0 where the axis is clamped (adjoint only)
};

// cell index and fraction from the compensated coordinate
// The cell index comes from rounding u = d/dx to the nearest integer with
// the float "magic number" 1.5*2^23 (two float adds and an integer subtract
// on the FP32/ALU pipes instead of floor + float-to-int conversions on the
// XU pipe); the fraction is then corrected into [0, 1).  Valid for |u| <
// 2^22, i.e. positions kept within the periodic box or a grid of < 4M cells;
// larger |u| takes the floorf path.
__device__ __forceinline__ bool axis32(const DevField& g, int a, float hi, float lo, AxF& o) {
    const float kMagic = 12582912.0f;  // 1.5 * 2^23
    float d = hi - g.x0f[a];
    float u = d * g.idxf[a];
    float fl;
    int i;
    if (fabsf(u) < 4194304.0f) {
        float tr = u + kMagic;
        i = __float_as_int(tr) - __float_as_int(kMagic);
        fl = tr - kMagic;
    } else {
        fl = floorf(u);
        i = (int)fl;
    }
    float rem = fmaf(-fl, g.dxf[a], d) + lo;
    float f = rem * g.idxf[a];
    if (f < 0.0f) {
        fl -= 1.0f;
        i -= 1;
        f += 1.0f;
    } else if (f >= 1.0f) {
        fl += 1.0f;
        i += 1;
        f -= 1.0f;
    }
    int na = g.n[a];
    if (g.bc == TP_BC_PERIODIC) {
        if (i >= na) i -= na;
        if (i < 0) i += na;
        if (i < 0 || i >= na) {  // far outside the box (positions not wrapped)
            i %= na;
            if (i < 0) i += na;
        }
        o.i0 = i;
        o.i1 = (i + 1 == na) ? 0 : i + 1;
        o.f = f;
        o.ds = g.idxf[a];
        return true;
    }
    float uc = fl + f;
    float umax = (float)(na - 1);
    o.ds = g.idxf[a];
    if (g.bc == TP_BC_CLAMP) {
        if (uc < 0.0f) {
            fl = 0.0f;
            f = 0.0f;
            o.ds = 0.0f;
        } else if (uc > umax) {
            fl = umax;
            f = 0.0f;
            o.ds = 0.0f;
        }
    } else if (!(uc >= 0.0f && uc <= umax)) {
        return false;
    }
    i = (int)fl;
    if (i > na - 2) {
        f += (float)(i - (na - 2));
        i = na - 2;
    }
    o.i0 = i;
    o.i1 = i + 1;
    o.f = f;
    return true;
}

__device__ __forceinline__ float lerp32(float a, float b, float f) { return fmaf(f, b - a, a); }

__device__ __forceinline__ F3 nanf3() {
    float q = __int_as_float(0x7fc00000);
    return {q, q, q};
}

__device__ __forceinline__ bool axes32(const DevField& g, const CPos& p, AxF& ax, AxF& ay, AxF& az) {
    bool ok = axis32(g, 0, p.hi[0], p.lo[0], ax);
    ok = axis32(g, 1, p.hi[1], p.lo[1], ay) && ok;
    ok = axis32(g, 2, p.hi[2], p.lo[2], az) && ok;
    return ok;
}

__device__ __forceinline__ F3 xyz(float4 q) { return {q.x, q.y, q.z}; }

// One 32-byte, 32-byte-aligned node record of the interleaved E/B table in a
// single 256-bit read-only load (sm_100 ld.global.nc.v8).
__device__ __forceinline__ void ldg_node8(const float4* p, float4& e, float4& b) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(e.x), "=f"(e.y), "=f"(e.z), "=f"(e.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// L2 policy: keep these lines in preference to others
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ F3 tri3(F3 v000, F3 v100, F3 v010, F3 v110, F3 v001, F3 v101, F3 v011,
                                   F3 v111, const AxF& ax, const AxF& ay, const AxF& az) {
    F3 o;
#define TPB_TRI32(c)                                                       \
    {                                                                      \
        float c0 = lerp32(lerp32(v000.c, v100.c, ax.f), lerp32(v010.c, v110.c, ax.f), ay.f); \
        float c1 = lerp32(lerp32(v001.c, v101.c, ax.f), lerp32(v011.c, v111.c, ax.f), ay.f); \
        o.c = lerp32(c0, c1, az.f);                                        \
    }
    TPB_TRI32(x)
    TPB_TRI32(y)
    TPB_TRI32(z)
#undef TPB_TRI32
    return o;
}

// quadratic fields: float64 evaluation of the compensated position, rounded
static __device__ __noinline__ F3 quad_eval32(const DevField& f, const CPos& p, double t) {
    double o[3];
    quad_eval(f, (double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
              (double)p.hi[2] + (double)p.lo[2], t, o);
    return {(float)o[0], (float)o[1], (float)o[2]};
}

// trilinear uniform-Cartesian grid (general grids: field_any32)
__device__ __forceinline__ F3 grid_eval32(const DevField& g, const CPos& p) {
    AxF ax, ay, az;
    if (!axes32(g, p, ax, ay, az)) return nanf3();
    const float4* T = g.tab32;
    const int nx = g.n[0], nxy = g.n[0] * g.n[1];
    int j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
    F3 v000 = xyz(__ldg(T + ax.i0 + j0 + k0)), v100 = xyz(__ldg(T + ax.i1 + j0 + k0));
    F3 v010 = xyz(__ldg(T + ax.i0 + j1 + k0)), v110 = xyz(__ldg(T + ax.i1 + j1 + k0));
    F3 v001 = xyz(__ldg(T + ax.i0 + j0 + k1)), v101 = xyz(__ldg(T + ax.i1 + j0 + k1));
    F3 v011 = xyz(__ldg(T + ax.i0 + j1 + k1)), v111 = xyz(__ldg(T + ax.i1 + j1 + k1));
    return tri3(v000, v100, v010, v110, v001, v101, v011, v111, ax, ay, az);
}

__device__ __forceinline__ F3 analytic_eval32(const DevField& f, const CPos& p, double t) {
    switch (f.kind) {
        case TP_FIELD_UNIFORM:
            return {f.vf[0], f.vf[1], f.vf[2]};
        case TP_FIELD_AFFINE: {
            float x = p.hi[0], y = p.hi[1], z = p.hi[2], tf = (float)t;
            return {f.vf[0] + f.Jf[0] * x + f.Jf[1] * y + f.Jf[2] * z + f.ratef[0] * tf,
                    f.vf[1] + f.Jf[3] * x + f.Jf[4] * y + f.Jf[5] * z + f.ratef[1] * tf,
                    f.vf[2] + f.Jf[6] * x + f.Jf[7] * y + f.Jf[8] * z + f.ratef[2] * tf};
        }
        case TP_FIELD_DIPOLE: {
            // unit-vector form keeps float intermediates normal:
            // B = K/r^3 (3 (mh.rh) rh - mh), K = coef |m|
            F3 d{(p.hi[0] - f.cf[0]) + p.lo[0], (p.hi[1] - f.cf[1]) + p.lo[1],
                 (p.hi[2] - f.cf[2]) + p.lo[2]};
            F3 mh{f.mhatf[0], f.mhatf[1], f.mhatf[2]};
            float ir = __frsqrt_rn(dot(d, d));  // correctly rounded: |rh| = 1 to 1 ulp
            F3 rh = ir * d;
            float mr = dot(mh, rh);
            float k = f.Kf * ir * ir * ir;
            return {k * (3.0f * mr * rh.x - mh.x), k * (3.0f * mr * rh.y - mh.y), k * (3.0f * mr * rh.z - mh.z)};
        }
        default:
            return {0.0f, 0.0f, 0.0f};
    }
}

template <bool PACKED_ONLY = false>
__device__ __forceinline__ void eval_EB32(const DevFields& F, const CPos& p, double t, F3& E, F3& B) {
    if (PACKED_ONLY || F.eb32) {
        AxF ax, ay, az;
        if (!axes32(F.B, p, ax, ay, az)) {
            E = nanf3();
            B = E;
            return;
        }
        const float4* T = F.eb32;
        const int nx = F.B.n[0], nxy = F.B.n[0] * F.B.n[1];
        int j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
        int n000 = 2 * (ax.i0 + j0 + k0), n100 = 2 * (ax.i1 + j0 + k0);
        int n010 = 2 * (ax.i0 + j1 + k0), n110 = 2 * (ax.i1 + j1 + k0);
        int n001 = 2 * (ax.i0 + j0 + k1), n101 = 2 * (ax.i1 + j0 + k1);
        int n011 = 2 * (ax.i0 + j1 + k1), n111 = 2 * (ax.i1 + j1 + k1);
        // 8 corners, each one aligned 32-byte sector (E xyz0, B xyz0) read by
        // one 256-bit load; all issued before any use
        float4 e000, b000, e100, b100, e010, b010, e110, b110;
        float4 e001, b001, e101, b101, e011, b011, e111, b111;
        ldg_node8(T + n000, e000, b000);
        ldg_node8(T + n100, e100, b100);
        ldg_node8(T + n010, e010, b010);
        ldg_node8(T + n110, e110, b110);
        ldg_node8(T + n001, e001, b001);
        ldg_node8(T + n101, e101, b101);
        ldg_node8(T + n011, e011, b011);
        ldg_node8(T + n111, e111, b111);
        E = tri3(xyz(e000), xyz(e100), xyz(e010), xyz(e110), xyz(e001), xyz(e101), xyz(e011),
                 xyz(e111), ax, ay, az);
        B = tri3(xyz(b000), xyz(b100), xyz(b010), xyz(b110), xyz(b001), xyz(b101), xyz(b011),
                 xyz(b111), ax, ay, az);
        return;
    }
    E = (F.E.kind == TP_FIELD_GRID) ? grid_eval32(F.E, p)
        : (F.E.kind == TP_FIELD_QUADRATIC) ? quad_eval32(*F.E.self, p, t) : analytic_eval32(F.E, p, t);
    B = (F.B.kind == TP_FIELD_GRID) ? grid_eval32(F.B, p)
        : (F.B.kind == TP_FIELD_QUADRATIC) ? quad_eval32(*F.B.self, p, t) : analytic_eval32(F.B, p, t);
}

// a series snapshot (never a series) in the FP32C arithmetic: trilinear
// grids through the float table as in grid_eval32, general grids through
// grid_general.cuh over the float table (out of line), quadratic and
// analytic fields as elsewhere
static __device__ __noinline__ F3 snapshot_general32(const DevField& g, const CPos& p) {
    double r[3] = {(double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
                   (double)p.hi[2] + (double)p.lo[2]};
    double o[3];
    if (!grid_general_eval<double, true>(g, r, o)) return nanf3();
    return {(float)o[0], (float)o[1], (float)o[2]};
}

__device__ __forceinline__ F3 snapshot_eval32(const DevField& g, const CPos& p, double t) {
    if (g.kind == TP_FIELD_GRID) return g.general ? snapshot_general32(g, p) : grid_eval32(g, p);
    if (g.kind == TP_FIELD_QUADRATIC) {
        double o[3];
        quad_eval(g, (double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
                  (double)p.hi[2] + (double)p.lo[2], t, o);
        return {(float)o[0], (float)o[1], (float)o[2]};
    }
    return analytic_eval32(g, p, t);
}

// time series (LazyTimeInterpolator, src/utility/interpolation.jl:337-430)
// in the FP32C arithmetic: the snapshot index and the weight w from the
// float64 times, the snapshots evaluated over their float tables (half the
// bytes of the float64 tables the FP64 kernels read) and blended in float,
// (1 - w) F_k + w F_{k+1}
static __device__ __noinline__ F3 series_eval32(const DevField& f, const CPos& p, double t) {
    const int k = series_index(f, t);
    if (k == 0) return snapshot_eval32(f.snaps[0], p, t);
    if (k >= f.nts) return snapshot_eval32(f.snaps[f.nts - 1], p, t);
    const double t1 = __ldg(f.ts + k - 1), t2 = __ldg(f.ts + k);
    const float w = (float)((t - t1) / (t2 - t1)), u = 1.0f - w;
    const F3 a = snapshot_eval32(f.snaps[k - 1], p, t), b = snapshot_eval32(f.snaps[k], p, t);
    return {u * a.x + w * b.x, u * a.y + w * b.y, u * a.z + w * b.z};
}

// E and B of the FP32C kernels for general grids and series (any field
// kind), out of line: one call evaluates both fields from their descriptors'
// device copies.  Measured on the config-2 field on a cubic grid, this is
// 1.3x the rate of one call per field; the float64 kernels keep one call per
// field (grid_general64), which measured 1.5x the rate of a combined call.
struct EB32 {
    F3 E, B;
};

__device__ __forceinline__ F3 field_any32(const DevField& f, const CPos& p, double t) {
    if (f.kind == TP_FIELD_GRID) {
        if (f.general) {
            double r[3] = {(double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
                           (double)p.hi[2] + (double)p.lo[2]};
            double o[3];
            if (!grid_general_eval<double, true>(f, r, o)) return nanf3();
            return {(float)o[0], (float)o[1], (float)o[2]};
        }
        return grid_eval32(f, p);
    }
    if (f.kind == TP_FIELD_QUADRATIC) {
        double o[3];
        quad_eval(f, (double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
                  (double)p.hi[2] + (double)p.lo[2], t, o);
        return {(float)o[0], (float)o[1], (float)o[2]};
    }
    if (f.kind == TP_FIELD_SERIES) return series_eval32(f, p, t);
    return analytic_eval32(f, p, t);
}

static __device__ __noinline__ EB32 eval_EB_any32(const DevField& Ef, const DevField& Bf, CPos p, double t) {
    EB32 o;
    o.E = field_any32(Ef, p, t);
    o.B = field_any32(Bf, p, t);
    return o;
}

template <int FK>
__device__ __forceinline__ void eval_EB32t(const DevFields& F, const CPos& p, double t, F3& E, F3& B) {
    if (FK == FK_ANALYTIC) {
        E = analytic_eval32(F.E, p, t);
        B = analytic_eval32(F.B, p, t);
    } else if (FK == FK_EBGRID) {
        eval_EB32<true>(F, p, t, E, B);
    } else if (FK == FK_GENGRID) {
        EB32 o = eval_EB_any32(*F.E.self, *F.B.self, p, t);
        E = o.E;
        B = o.B;
    } else {
        eval_EB32<false>(F, p, t, E, B);
    }
}

__device__ __forceinline__ bool fields_static32(const DevFields& F) {
    bool e = !((F.E.kind == TP_FIELD_AFFINE || F.E.kind == TP_FIELD_QUADRATIC) &&
               (F.E.rate[0] != 0.0 || F.E.rate[1] != 0.0 || F.E.rate[2] != 0.0));
    bool b = !((F.B.kind == TP_FIELD_AFFINE || F.B.kind == TP_FIELD_QUADRATIC) &&
               (F.B.rate[0] != 0.0 || F.B.rate[1] != 0.0 || F.B.rate[2] != 0.0));
    return e && b && F.E.kind != TP_FIELD_SERIES && F.B.kind != TP_FIELD_SERIES;
}

// ---------------------------------------------------------------- updates
// Velocity as a compensated float pair, v = h + l, advanced in "delta form":
// the kernels compute the change dv = v_new - v in float (|dv| ~ the
// rotation angle times |v|, so its rounding is ~1e-8 |v|) and add it with
// TwoSum.  The scalar rotation coefficients -- the only quantities whose
// float rounding would bias the gyrophase every step -- are formed in
// float64 from the float rotation vector; 1/(1+|t|^2) and 1/A use a float
// reciprocal refined by one float64 Newton step.
struct CV {
    F3 h, l;
};

__device__ __forceinline__ void cv_add(CV& v, F3 d) {
    cadd(v.h.x, v.l.x, d.x);
    cadd(v.h.y, v.l.y, d.y);
    cadd(v.h.z, v.l.z, d.z);
}

__device__ __forceinline__ CV cv_from(const double* u) {
    CV v;
    v.h = {(float)u[0], (float)u[1], (float)u[2]};
    v.l = {(float)(u[0] - (double)v.h.x), (float)(u[1] - (double)v.h.y), (float)(u[2] - (double)v.h.z)};
    return v;
}

// Boris (boris.jl:19-31): dv = 2 h E + (v- + v- x t) x s,  h = q2m*dt/2,
// s = 2 t / (1 + |t|^2) with a correctly rounded reciprocal
__device__ __forceinline__ F3 boris_delta32(F3 v, F3 E, F3 B, float h) {
    F3 t = h * B;
    float sc = 2.0f * __frcp_rn(1.0f + dot(t, t));
    F3 he = h * E;
    F3 vm = v + he;
    F3 vp = vm + cross(vm, t);
    F3 d = cross(vp, sc * t);
    return d + (2.0f * he);
}

// Multistep / Hyper Boris (multistep_boris.jl:65-142) in closed form,
// fac = q2m*dt/(2n):
//   dv = (c1 - 1) v + c2 v x t + c3 (v.t) t + c2 e + c3 e x t + c6 (e.t) t
// with c1 - 1 = -2 s q^2 / A = -s c3 (because zr^2 + s q^2 = |1 + i tau|^(2n) = A),
// so no coefficient is formed by cancellation.
__device__ __forceinline__ F3 multistep_delta32(F3 v, F3 E, F3 B, float fac, int N, int n) {
    F3 t_n = fac * B;
    F3 e_n = fac * E;
    float s = dot(t_n, t_n);
    if (N != 2) {
        float f_N, e_corr;
        if (N == 4) {
            f_N = 1.0f + s * (1.0f / 3.0f);
            e_corr = -1.0f / 3.0f;
        } else {
            f_N = 1.0f + s * (1.0f / 3.0f) + 2.0f * s * s * (1.0f / 15.0f);
            e_corr = -1.0f / 3.0f - 2.0f * s * (1.0f / 15.0f);
        }
        float edt = dot(e_n, t_n);
        e_n = f_N * e_n + (e_corr * edt) * t_n;
        t_n = f_N * t_n;
        s = dot(t_n, t_n);
    }
    float zr = 1.0f, q = 0.0f, A = 1.0f, R = 0.0f;
    for (int k = 0; k < n; ++k) {
        R = R + (float)(k + 1) * A + 2.0f * q * q + zr * q;
        float nzr = zr - s * q;
        q = zr + q;
        zr = nzr;
        A = A * (1.0f + s);
    }
    float invA = __frcp_rn(A);
    float c2 = 2.0f * zr * q * invA;
    float c3 = 2.0f * q * q * invA;
    float c6 = 2.0f * R * invA;
    float c1m1 = -s * c3;
    float vdt = dot(v, t_n), edt = dot(e_n, t_n);
    F3 vxt = cross(v, t_n), ext = cross(e_n, t_n);
    return c1m1 * v + c2 * vxt + (c3 * vdt) * t_n + c2 * e_n + c3 * ext + (c6 * edt) * t_n;
}

// the float factor of a velocity update of length dt: q2m*dt/2 (Boris) or
// q2m*dt/(2n) (Multistep), rounded once from float64
template <bool MULTI>
__device__ __forceinline__ float vfac(const BorisArgs& a, double dt) {
    return MULTI ? (float)(a.q2m * dt / (double)(2 * a.nsub)) : (float)(a.q2m * 0.5 * dt);
}

// v advanced by one velocity update with factor h (see vfac) and fields (E, B)
template <bool MULTI>
__device__ __forceinline__ CV vel32h(CV v, F3 E, F3 B, const BorisArgs& a, float h) {
    F3 d = MULTI ? multistep_delta32(v.h, E, B, h, a.order, a.nsub) : boris_delta32(v.h, E, B, h);
    cv_add(v, d);
    return v;
}

template <bool MULTI>
__device__ __forceinline__ CV vel32(CV v, F3 E, F3 B, const BorisArgs& a, double dt) {
    return vel32h<MULTI>(v, E, B, a, vfac<MULTI>(a, dt));
}

// position push x += v dt with dt = dth + dtl (float pair)
__device__ __forceinline__ void cpos_push_cv(const BorisArgs& a, CPos& p, const CV& v, float dth, float dtl) {
    F3 d{fmaf(v.h.x, dth, fmaf(v.h.x, dtl, v.l.x * dth)), fmaf(v.h.y, dth, fmaf(v.h.y, dtl, v.l.y * dth)),
         fmaf(v.h.z, dth, fmaf(v.h.z, dtl, v.l.z * dth))};
    cpos_push(a, p, d, 1.0f);
}

// ---------------------------------------------------------------- analytic fields: invariant-preserving update
// With analytic fields (FK_ANALYTIC) the FP32C kernels keep the rotation
// factors of the closed form in float, but the rotation axis, the velocity
// and the field in float64.  The float delta form above leaves two random
// walks that dominate the final-position error of long orbits in a dipole:
//   |v|       the float rounding of each increment (~eps_f * angle per step)
//             walks the energy, which shifts bounce and drift phases;
//   pitch     the float field's direction error (~6e-8 rad per evaluation)
//             tilts every rotation axis, which walks v . b and with it the
//             magnetic moment and the mirror points.
// Rotation factors rounded in float only misplace the gyrophase, but their
// mutual consistency is what conserves |v| and v . t: one float64 step
// restores (1 + c1)^2 + c2^2 |t|^2 = 1 (a common scale of 1 + c1 and c2) and
// c1 + c3 |t|^2 = 0 (c3 alone), after which the update is orthogonal on
// float64's scale.  The field costs about thirty float64 operations: 1/r from
// a float rsqrt and one float64 Newton step (no sqrt, no division).

// position of a compensated pair in float64 (analytic fields: no wrapping)
__device__ __forceinline__ D3 cpos_d3(const CPos& p) {
    return {(double)p.hi[0] + (double)p.lo[0], (double)p.hi[1] + (double)p.lo[1],
            (double)p.hi[2] + (double)p.lo[2]};
}

// analytic field in float64 at a compensated position
__device__ __forceinline__ D3 analytic_eval_mixed(const DevField& f, const CPos& p, double t) {
    switch (f.kind) {
        case TP_FIELD_UNIFORM:
            return {f.v[0], f.v[1], f.v[2]};
        case TP_FIELD_AFFINE: {
            const D3 r = cpos_d3(p);
            return {f.v[0] + f.J[0] * r.x + f.J[1] * r.y + f.J[2] * r.z + f.rate[0] * t,
                    f.v[1] + f.J[3] * r.x + f.J[4] * r.y + f.J[5] * r.z + f.rate[1] * t,
                    f.v[2] + f.J[6] * r.x + f.J[7] * r.y + f.J[8] * r.z + f.rate[2] * t};
        }
        case TP_FIELD_DIPOLE: {
            // B = coef (3 (m.d) d / r^5 - m / r^3), 1/r = y (1.5 - r^2 y^2 / 2)
            // from the float estimate y (relative error ~1e-13 after the step)
            const D3 d = cpos_d3(p) - D3{f.c[0], f.c[1], f.c[2]};
            const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
            double y = (double)rsqrtf((float)r2);
            y = y * fma(-0.5 * r2, y * y, 1.5);
            const double ir2 = y * y;
            const double k3 = f.coef * (ir2 * y);
            const double k5 = 3.0 * (k3 * ir2) * (f.m[0] * d.x + f.m[1] * d.y + f.m[2] * d.z);
            return {k5 * d.x - k3 * f.m[0], k5 * d.y - k3 * f.m[1], k5 * d.z - k3 * f.m[2]};
        }
        default:
            return {0.0, 0.0, 0.0};
    }
}

// Multistep / Hyper Boris (multistep_boris.jl:65-142) -- and Boris itself,
// which is its n = 1, N = 2 case (c1 + 1 = c2 = c3 = c6 = 2 / (1 + |t|^2)) --
// with fac = q2m dt / (2n): float rotation factors from the float copy of
// the axis, refined as above, applied in float64.
__device__ __forceinline__ D3 rot_mixed(D3 v, D3 E, D3 B, double fac, int N, int n, bool hasE) {
    D3 t = fac * B;
    D3 e = hasE ? fac * E : D3{0.0, 0.0, 0.0};
    double sd = dot(t, t);
    float s = (float)sd;
    if (N != 2) {
        float f_N, e_corr;
        if (N == 4) {
            f_N = 1.0f + s * (1.0f / 3.0f);
            e_corr = -1.0f / 3.0f;
        } else {
            f_N = 1.0f + s * (1.0f / 3.0f) + 2.0f * s * s * (1.0f / 15.0f);
            e_corr = -1.0f / 3.0f - 2.0f * s * (1.0f / 15.0f);
        }
        const double fd = f_N;
        if (hasE) e = fd * e + ((double)e_corr * dot(e, t)) * t;
        t = fd * t;
        sd = (fd * fd) * sd;
        s = (float)sd;
    }
    float zr = 1.0f, q = 0.0f, A = 1.0f, R = 0.0f;
    for (int k = 0; k < n; ++k) {
        R = R + (float)(k + 1) * A + 2.0f * q * q + zr * q;
        float nzr = zr - s * q;
        q = zr + q;
        zr = nzr;
        A = A * (1.0f + s);
    }
    // 1/A: the float estimate and one float64 Newton step
    double invA = (double)__fdividef(1.0f, A);
    invA = invA * fma(-(double)A, invA, 2.0);
    double C2 = (2.0 * zr) * q * invA;
    double C3 = (2.0 * q) * q * invA;
    double C1 = -(double)s * C3;
    // consistency in float64: scale (1 + C1, C2) onto the unit circle, then
    // C3 from C1 + C3 |t|^2 = 0
    const double hg = 0.5 * fma(C1, 2.0 + C1, C2 * C2 * sd);
    C1 = C1 - hg * (1.0 + C1);
    C2 = C2 - hg * C2;
    const float rs = s > 0.0f ? __fdividef(1.0f, s) : 0.0f;
    C3 = C3 - fma(C3, sd, C1) * (double)rs;
    const D3 vxt = cross(v, t);
    D3 dv = C1 * v + C2 * vxt + (C3 * dot(v, t)) * t;
    if (hasE) {
        const double c6 = (2.0 * R) * invA;
        dv = dv + C2 * e + C3 * cross(e, t) + (c6 * dot(e, t)) * t;
    }
    return v + dv;
}

// velocity update of length dt, fields (E, B) in float64
template <bool MULTI>
__device__ __forceinline__ D3 vel_mixed(D3 v, D3 E, D3 B, const BorisArgs& a, double dt) {
    const bool hasE = a.f.E.kind != TP_FIELD_ZERO;
    if (MULTI) return rot_mixed(v, E, B, a.q2m * dt / (double)(2 * a.nsub), a.order, a.nsub, hasE);
    return rot_mixed(v, E, B, a.q2m * 0.5 * dt, 2, 1, hasE);
}

// position push x += v dt from a float64 velocity
__device__ __forceinline__ void cpos_push_d(const BorisArgs& a, CPos& p, const D3& v, double dt) {
    const F3 d{(float)(v.x * dt), (float)(v.y * dt), (float)(v.z * dt)};
    cpos_push<false>(a, p, d, 1.0f);
}

// ---------------------------------------------------------------- velocity representation per field kind
// Grids: compensated float velocity, float fields, delta form.  Analytic
// fields: float64 velocity and fields, invariant-preserving update.
template <int FK>
struct Vel32 {
    using V = CV;
    using Fv = F3;
    static __device__ __forceinline__ V init(const double* u) { return cv_from(u); }
    static __device__ __forceinline__ double comp(const V& v, int c) {
        return c == 0 ? (double)v.h.x + (double)v.l.x : (c == 1 ? (double)v.h.y + (double)v.l.y
                                                                 : (double)v.h.z + (double)v.l.z);
    }
    static __device__ __forceinline__ bool has_nan(const V& v) {
        return isnan(v.h.x) || isnan(v.h.y) || isnan(v.h.z);
    }
    static __device__ __forceinline__ void fields(const DevFields& F, const CPos& p, double t, Fv& E, Fv& B) {
        eval_EB32t<FK>(F, p, t, E, B);
    }
    using H = float;  // factor of one velocity update
    template <bool MULTI>
    static __device__ __forceinline__ H fac(const BorisArgs& a, double dt) {
        return vfac<MULTI>(a, dt);
    }
    template <bool MULTI>
    static __device__ __forceinline__ V step_h(const V& v, const Fv& E, const Fv& B, const BorisArgs& a, H h) {
        return vel32h<MULTI>(v, E, B, a, h);
    }
    template <bool MULTI>
    static __device__ __forceinline__ V step(const V& v, const Fv& E, const Fv& B, const BorisArgs& a, double dt) {
        return vel32<MULTI>(v, E, B, a, dt);
    }
    static __device__ __forceinline__ void push(const BorisArgs& a, CPos& p, const V& v, float dth, float dtl,
                                                double) {
        cpos_push_cv(a, p, v, dth, dtl);
    }
    static __device__ __forceinline__ double bmag2(const Fv& B) { return (double)dot(B, B); }
    static __device__ __forceinline__ double fcomp(const Fv& f, int c) { return c == 0 ? f.x : (c == 1 ? f.y : f.z); }
};

template <>
struct Vel32<FK_ANALYTIC> {
    using V = D3;
    using Fv = D3;
    static __device__ __forceinline__ V init(const double* u) { return {u[0], u[1], u[2]}; }
    static __device__ __forceinline__ double comp(const V& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
    static __device__ __forceinline__ bool has_nan(const V& v) { return isnan(v.x) || isnan(v.y) || isnan(v.z); }
    static __device__ __forceinline__ void fields(const DevFields& F, const CPos& p, double t, Fv& E, Fv& B) {
        E = analytic_eval_mixed(F.E, p, t);
        B = analytic_eval_mixed(F.B, p, t);
    }
    using H = double;
    template <bool MULTI>
    static __device__ __forceinline__ H fac(const BorisArgs& a, double dt) {
        return MULTI ? a.q2m * dt / (double)(2 * a.nsub) : a.q2m * 0.5 * dt;
    }
    template <bool MULTI>
    static __device__ __forceinline__ V step_h(const V& v, const Fv& E, const Fv& B, const BorisArgs& a, H h) {
        const bool hasE = a.f.E.kind != TP_FIELD_ZERO;
        return MULTI ? rot_mixed(v, E, B, h, a.order, a.nsub, hasE) : rot_mixed(v, E, B, h, 2, 1, hasE);
    }
    template <bool MULTI>
    static __device__ __forceinline__ V step(const V& v, const Fv& E, const Fv& B, const BorisArgs& a, double dt) {
        return vel_mixed<MULTI>(v, E, B, a, dt);
    }
    static __device__ __forceinline__ void push(const BorisArgs& a, CPos& p, const V& v, float, float, double dt) {
        cpos_push_d(a, p, v, dt);
    }
    static __device__ __forceinline__ double bmag2(const Fv& B) { return dot(B, B); }
    static __device__ __forceinline__ double fcomp(const Fv& f, int c) { return c == 0 ? f.x : (c == 1 ? f.y : f.z); }
};

}  // namespace

}  // namespace tpb
