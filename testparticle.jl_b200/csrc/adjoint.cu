// adjoint.cu -- discrete adjoint of the fixed-step Boris map, in the FP32C
// arithmetic of boris_fp32c.cu (compensated positions and velocities).
//
// The map (boris.jl:445-557 without saves or termination):
//   v_{-1/2} = U(v_0, x_0, -dt/2);  for k = 0..N-1:
//   v_{k+1/2} = U(v_{k-1/2}, x_k, dt),  x_{k+1} = x_k + dt v_{k+1/2};
//   v_N = U(v_{N-1/2}, x_N, dt_final)
// with U the Boris velocity update (boris.jl:19-45), in delta form
//   U(v) = v + 2hE + vp x s,  vm = v + hE,  vp = vm + vm x t,  t = hB,
//   s = sc t,  sc = 2 / (1 + |t|^2),  h = q2m * dt_u / 2.
//
// Forward (k_adj_forward): the push of k_fixed32c, writing the compensated
// state every K steps to the tape and the final save to u_final.
//
// Backward (k_adj_backward): one thread per particle walks the checkpoint
// segments from last to first.  Each segment is recomputed from its
// checkpoint with the forward's own arithmetic (so the recomputed states are
// the forward's bit for bit), each step's input state going to a record
// buffer, and then the records are run backwards through the adjoint of one
// step: with lo the cotangent of v_{k+1/2} including the position update
// (lo = lv + dt lx), the adjoint of U is (c = a x b gives la += b x lc,
// lb += lc x a)
//   ls = lo x vp,  lvp = s x lo,  lvm = lvp + t x lvp,
//   lt = lvp x vm + sc ls - sc^2 (t . ls) t,
//   lv_in = lo + lvm,  lE = h (2 lo + lvm),  lB = h lt.
// E and B depend on x and on the node values through the trilinear weights
// w_c(x): node c receives w_c lE and w_c lB (red.global.add.v4.f32 into a
// gradient table laid out like the field table), and
// lx += sum_c grad w_c(x) (E_c . lE + B_c . lB).
// Analytic fields contribute J^T l to lx (J the field's Jacobian) and their
// parameter gradient (uniform offset, or dipole moment) to g_param.
//
// Range.  In a chaotic field the cotangents grow exponentially with the
// number of steps (in the 128^3 turbulent field, |dx_N/dx_0| reaches 1e18 to
// 1e27 after 4096 steps), beyond float32.  Each particle therefore carries
// its cotangent as float32 values times 2^e (renormalised by exact powers of
// two), and the node-gradient tables hold float32 values times 2^G, one G per
// pass.  A pass whose largest node contribution would not fit reports the
// exponent it needed (A.need) and the host repeats it with a larger G.
#include <climits>

#include "fp32c_common.cuh"
#include "tp_device.cuh"
#include "tp_launch.h"

namespace tpb {

namespace {

constexpr int kRec = 9;   // record words per particle-step

__device__ __forceinline__ F3 nanf3_() { return nanf3(); }

// Checkpoint: position hi xyz, lo xyz, velocity hi xyz, lo xyz.  The wrap
// counts are left out: the backward evaluates fields only, and wrapped axes
// are periodic in every field.  Written and read once, with streaming
// (evict-first) hints so that the tape does not displace the field table
// from L2.
__device__ __forceinline__ void store_ck(const AdjArgs& A, int64_t s, int64_t i, const CPos& p, const CV& v) {
    const int64_t n = A.a.n;
    float* c = A.ckpt + s * kAdjCkWords * n + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        __stcs(c + (0 + k) * n, p.hi[k]);
        __stcs(c + (3 + k) * n, p.lo[k]);
    }
    __stcs(c + 6 * n, v.h.x);
    __stcs(c + 7 * n, v.h.y);
    __stcs(c + 8 * n, v.h.z);
    __stcs(c + 9 * n, v.l.x);
    __stcs(c + 10 * n, v.l.y);
    __stcs(c + 11 * n, v.l.z);
}

__device__ __forceinline__ void load_ck(const AdjArgs& A, int64_t s, int64_t i, CPos& p, CV& v) {
    const int64_t n = A.a.n;
    const float* c = A.ckpt + s * kAdjCkWords * n + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.hi[k] = __ldcs(c + (0 + k) * n);
        p.lo[k] = __ldcs(c + (3 + k) * n);
        p.w[k] = 0;
    }
    v.h = {__ldcs(c + 6 * n), __ldcs(c + 7 * n), __ldcs(c + 8 * n)};
    v.l = {__ldcs(c + 9 * n), __ldcs(c + 10 * n), __ldcs(c + 11 * n)};
}

__device__ __forceinline__ void store_rec(const AdjArgs& A, int j, int64_t i, const CPos& p, F3 v) {
    const int64_t n = A.a.n;
    float* r = A.rec + (int64_t)j * kRec * n + i;
    r[0] = p.hi[0];
    r[n] = p.hi[1];
    r[2 * n] = p.hi[2];
    r[3 * n] = p.lo[0];
    r[4 * n] = p.lo[1];
    r[5 * n] = p.lo[2];
    r[6 * n] = v.x;
    r[7 * n] = v.y;
    r[8 * n] = v.z;
}

// the wrap counts are not needed to evaluate a field (wrapped axes are
// periodic in every field), so records leave them out
__device__ __forceinline__ void load_rec(const AdjArgs& A, int j, int64_t i, CPos& p, F3& v) {
    const int64_t n = A.a.n;
    const float* r = A.rec + (int64_t)j * kRec * n + i;
    p.hi[0] = r[0];
    p.hi[1] = r[n];
    p.hi[2] = r[2 * n];
    p.lo[0] = r[3 * n];
    p.lo[1] = r[4 * n];
    p.lo[2] = r[5 * n];
    p.w[0] = p.w[1] = p.w[2] = 0;
    v = {r[6 * n], r[7 * n], r[8 * n]};
}

// ------------------------------------------------------------ adjoint of U
struct UAdj {
    F3 lv, lE, lB;
};

// vm = v + hE, the update's half-accelerated velocity
__device__ __forceinline__ F3 vminus(F3 v, F3 E, float h) {
    F3 he = h * E;
    return v + he;
}

// The adjoint depends on v and E only through vm (lE = h (2 lo + lvm) holds
// for any E), so records of the fused backward keep vm instead of both.
__device__ __forceinline__ UAdj u_adjoint_vm(F3 vm, F3 B, float h, F3 lo) {
    F3 t = h * B;
    float sc = 2.0f * __frcp_rn(1.0f + dot(t, t));
    F3 vp = vm + cross(vm, t);
    F3 s = sc * t;
    F3 ls = cross(lo, vp);
    F3 lvp = cross(s, lo);
    F3 lvm = lvp + cross(t, lvp);
    F3 lt = cross(lvp, vm) + sc * ls - (sc * sc * dot(t, ls)) * t;
    UAdj r;
    r.lv = lo + lvm;
    r.lE = h * ((2.0f * lo) + lvm);
    r.lB = h * lt;
    return r;
}

__device__ __forceinline__ UAdj u_adjoint(F3 v, F3 E, F3 B, float h, F3 lo) {
    return u_adjoint_vm(vminus(v, E, h), B, h, lo);
}

// ------------------------------------------------------- trilinear stencil
// corners in the order 000, 100, 010, 110, 001, 101, 011, 111 (x fastest)
__device__ __forceinline__ void tri_nodes(const DevField& g, const AxF& ax, const AxF& ay, const AxF& az,
                                          int* nd) {
    const int nx = g.n[0], nxy = g.n[0] * g.n[1];
    const int j0 = ay.i0 * nx, j1 = ay.i1 * nx, k0 = az.i0 * nxy, k1 = az.i1 * nxy;
    nd[0] = ax.i0 + j0 + k0;
    nd[1] = ax.i1 + j0 + k0;
    nd[2] = ax.i0 + j1 + k0;
    nd[3] = ax.i1 + j1 + k0;
    nd[4] = ax.i0 + j0 + k1;
    nd[5] = ax.i1 + j0 + k1;
    nd[6] = ax.i0 + j1 + k1;
    nd[7] = ax.i1 + j1 + k1;
}

__device__ __forceinline__ void tri_weights(const AxF& ax, const AxF& ay, const AxF& az, float* w) {
    const float x0 = 1.0f - ax.f, x1 = ax.f, y0 = 1.0f - ay.f, y1 = ay.f, z0 = 1.0f - az.f, z1 = az.f;
    const float a00 = y0 * z0, a10 = y1 * z0, a01 = y0 * z1, a11 = y1 * z1;
    w[0] = x0 * a00;
    w[1] = x1 * a00;
    w[2] = x0 * a10;
    w[3] = x1 * a10;
    w[4] = x0 * a01;
    w[5] = x1 * a01;
    w[6] = x0 * a11;
    w[7] = x1 * a11;
}

__device__ __forceinline__ void red_add3(float4* p, float a, float b, float c) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(0.0f)
                 : "memory");
}

// the same with an L2 eviction-priority policy
__device__ __forceinline__ void red_add3(float4* p, float a, float b, float c, uint64_t pol) {
    asm volatile("red.global.add.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(a), "f"(b),
                 "f"(c), "f"(0.0f), "l"(pol)
                 : "memory");
}

// Scatter w_c * la (and w_c * lb when NV == 2) to the 8 corner nodes of a
// gradient table with NV float4 entries per node.  Warp aggregation: lanes
// whose particles sit in the same cell update the same 8 nodes, so
//  * when no two lanes share a cell (the usual case) every lane adds its own;
//  * when the whole warp shares one cell, a butterfly sum leaves one
//    red.global.add per node and vector;
//  * for groups of 4 or more lanes the group's lowest lane pulls the others'
//    contributions by shuffles and adds the group sum;
//  * small groups add individually (the adds are atomic either way).
#define RED3(p, a, b, c) (POL ? red_add3(p, a, b, c, pol) : red_add3(p, a, b, c))
template <int NV, bool POL = false>
__device__ __forceinline__ void scatter(float4* G, const int* nd, const float* w, F3 la, F3 lb,
                                        uint64_t pol = 0) {
    const unsigned act = __activemask();
    const unsigned me = 1u << (threadIdx.x & 31);
    const unsigned peers = __match_any_sync(act, nd[0]);
    const int gsize = __popc(peers);
    const int gmax = __reduce_max_sync(act, (unsigned)gsize);
    if (gmax == 1) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            RED3(G + (int64_t)NV * nd[c], w[c] * la.x, w[c] * la.y, w[c] * la.z);
            if (NV == 2) RED3(G + 2 * (int64_t)nd[c] + 1, w[c] * lb.x, w[c] * lb.y, w[c] * lb.z);
        }
        return;
    }
    if (act == 0xffffffffu && gsize == 32) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float q[6] = {w[c] * la.x, w[c] * la.y, w[c] * la.z, w[c] * lb.x, w[c] * lb.y, w[c] * lb.z};
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int k = 0; k < 3 * NV; ++k) q[k] += __shfl_xor_sync(0xffffffffu, q[k], o);
            if (me == 1u) {
                RED3(G + (int64_t)NV * nd[c], q[0], q[1], q[2]);
                if (NV == 2) RED3(G + 2 * (int64_t)nd[c] + 1, q[3], q[4], q[5]);
            }
        }
        return;
    }
    if (gmax >= 4) {
        const bool leader = (peers & (0u - peers)) == me;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float q[6] = {w[c] * la.x, w[c] * la.y, w[c] * la.z, w[c] * lb.x, w[c] * lb.y, w[c] * lb.z};
            float acc[6] = {q[0], q[1], q[2], q[3], q[4], q[5]};
            unsigned rest = peers & (peers - 1u);  // the group without its lowest lane
            for (int r = 1; r < gmax; ++r) {
                const bool have = rest != 0u;
                const int src = have ? __ffs(rest) - 1 : (int)(threadIdx.x & 31);
                rest &= rest - 1u;
#pragma unroll
                for (int k = 0; k < 3 * NV; ++k) {
                    float x = __shfl_sync(act, q[k], src);
                    if (have) acc[k] += x;
                }
            }
            if (leader) {
                RED3(G + (int64_t)NV * nd[c], acc[0], acc[1], acc[2]);
                if (NV == 2) RED3(G + 2 * (int64_t)nd[c] + 1, acc[3], acc[4], acc[5]);
            }
        }
        return;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        RED3(G + (int64_t)NV * nd[c], w[c] * la.x, w[c] * la.y, w[c] * la.z);
        if (NV == 2) RED3(G + 2 * (int64_t)nd[c] + 1, w[c] * lb.x, w[c] * lb.y, w[c] * lb.z);
    }
}

#undef RED3

// ----------------------------------------------------- cotangent frame
// lambda_true = lambda * 2^e; node contributions are scaled by f = 2^(e - G)
// (0 when they would underflow the table); mx is the largest exponent of a
// node contribution seen, e included.
struct Frame {
    int e;
    int mx;
    float f;
    double s;  // 2^e, for the float64 parameter accumulators
};

__device__ __forceinline__ int fexp(float m) { return ((__float_as_int(m) >> 23) & 0xff) - 127; }

__device__ __forceinline__ void frame_set(Frame& fr, int G) {
    const int d = fr.e - G;
    fr.f = d < -126 ? 0.0f : __int_as_float((min(d, 127) + 127) << 23);
    fr.s = ldexp(1.0, fr.e);
}

// keep max |lambda| near 1: exact rescaling by a power of two
__device__ __forceinline__ void renorm(F3& lx, F3& lv, Frame& fr, int G) {
    float m = fmaxf(fmaxf(fmaxf(fabsf(lx.x), fabsf(lx.y)), fmaxf(fabsf(lx.z), fabsf(lv.x))),
                    fmaxf(fabsf(lv.y), fabsf(lv.z)));
    int k = fexp(m);
    if ((k > 40 && k < 128) || (k < -40 && m > 0.0f)) {
        float sc = __int_as_float((127 - k) << 23);  // 2^-k, k in [-127, 127]
        lx = sc * lx;
        lv = sc * lv;
        fr.e += k;
        frame_set(fr, G);
    }
}

// value and Jacobian (d/dx, d/dy, d/dz of the three components) of the
// trilinear interpolant; the value uses the forward's lerp order
__device__ __forceinline__ void tri_val_jac(const float4* q, const AxF& ax, const AxF& ay, const AxF& az, F3& val,
                                            F3& dx, F3& dy, F3& dz) {
    val = tri3(xyz(q[0]), xyz(q[1]), xyz(q[2]), xyz(q[3]), xyz(q[4]), xyz(q[5]), xyz(q[6]), xyz(q[7]), ax, ay, az);
    const float fx = ax.f, fy = ay.f, fz = az.f;
#define TPB_JAC(c)                                                                                           \
    dx.c = lerp32(lerp32(q[1].c - q[0].c, q[3].c - q[2].c, fy), lerp32(q[5].c - q[4].c, q[7].c - q[6].c, fy), fz) * \
           ax.ds;                                                                                            \
    dy.c = lerp32(lerp32(q[2].c - q[0].c, q[3].c - q[1].c, fx), lerp32(q[6].c - q[4].c, q[7].c - q[5].c, fx), fz) * \
           ay.ds;                                                                                            \
    dz.c = lerp32(lerp32(q[4].c - q[0].c, q[5].c - q[1].c, fx), lerp32(q[6].c - q[2].c, q[7].c - q[3].c, fx), fy) * \
           az.ds;
    TPB_JAC(x)
    TPB_JAC(y)
    TPB_JAC(z)
#undef TPB_JAC
}

// J^T l for a Jacobian given by its columns (dx, dy, dz)
__device__ __forceinline__ F3 jt(const F3& dx, const F3& dy, const F3& dz, F3 l) {
    return {dot(dx, l), dot(dy, l), dot(dz, l)};
}

// node contributions: weights times the frame's scale, and the exponent record
__device__ __forceinline__ bool scale_weights(const AxF& ax, const AxF& ay, const AxF& az, F3 la, F3 lb,
                                              Frame& fr, float* w) {
    if (fr.f == 0.0f) return false;
    float m = fmaxf(fmaxf(fmaxf(fabsf(la.x), fabsf(la.y)), fmaxf(fabsf(la.z), fabsf(lb.x))),
                    fmaxf(fabsf(lb.y), fabsf(lb.z)));
    fr.mx = max(fr.mx, fexp(m) + fr.e);
    tri_weights(ax, ay, az, w);
#pragma unroll
    for (int c = 0; c < 8; ++c) w[c] *= fr.f;
    return true;
}

// --------------------------------------------- one step, interleaved E/B grid
// Returns the cotangent of the update's input velocity; adds the position
// cotangent to lx and scatters the node gradients.
__device__ __forceinline__ F3 adj_step_eb(const AdjArgs& A, const CPos& p, F3 v, float h, F3 lo, F3& lx,
                                          Frame& fr) {
    const DevFields& F = A.a.f;
    AxF ax, ay, az;
    if (!axes32(F.B, p, ax, ay, az)) {  // outside a FillExtrap(NaN) grid: NaN, as the forward
        lx = nanf3_();
        return nanf3_();
    }
    int nd[8];
    tri_nodes(F.B, ax, ay, az, nd);
    F3 E, B, Ex, Ey, Ez, Bx, By, Bz;
    {
        const float4* T = F.eb32;
        float4 e[8], b[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) ldg_node8(T + 2 * (int64_t)nd[c], e[c], b[c]);
        tri_val_jac(e, ax, ay, az, E, Ex, Ey, Ez);
        tri_val_jac(b, ax, ay, az, B, Bx, By, Bz);
    }
    UAdj u = u_adjoint(v, E, B, h, lo);
    lx = lx + jt(Ex, Ey, Ez, u.lE) + jt(Bx, By, Bz, u.lB);
    float w[8];
    if (scale_weights(ax, ay, az, u.lE, u.lB, fr, w)) scatter<2>(A.g_eb, nd, w, u.lE, u.lB);
    return u.lv;
}

// ------------------------------------------------ one step, generic fields
struct GridKeep {
    AxF ax, ay, az;
    int nd[8];
    F3 dx, dy, dz;
    bool ok;
};

// the arithmetic of grid_eval32, keeping the stencil and the Jacobian
__device__ __forceinline__ F3 grid_eval_keep(const DevField& g, const CPos& p, GridKeep& k) {
    k.ok = axes32(g, p, k.ax, k.ay, k.az);
    if (!k.ok) return nanf3_();
    tri_nodes(g, k.ax, k.ay, k.az, k.nd);
    float4 q[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) q[c] = __ldg(g.tab32 + k.nd[c]);
    F3 val;
    tri_val_jac(q, k.ax, k.ay, k.az, val, k.dx, k.dy, k.dz);
    return val;
}

// field f evaluated to lam's cotangent: lx += J^T lam, parameter gradient
// to th (analytic kinds), node gradients to G (grids)
__device__ __forceinline__ void field_adj(const DevField& f, const CPos& p, const GridKeep& k, F3 lam, float4* G,
                                          F3& lx, double* th, Frame& fr) {
    switch (f.kind) {
        case TP_FIELD_GRID: {
            if (!k.ok) {
                lx = nanf3_();
                return;
            }
            lx = lx + jt(k.dx, k.dy, k.dz, lam);
            float w[8];
            if (scale_weights(k.ax, k.ay, k.az, lam, lam, fr, w)) scatter<1>(G, k.nd, w, lam, lam);
            return;
        }
        case TP_FIELD_AFFINE: {
            // F = v + J x (static): d/dx = J, d/d(offset) = I
            const float* J = f.Jf;
            lx = lx + F3{J[0] * lam.x + J[3] * lam.y + J[6] * lam.z, J[1] * lam.x + J[4] * lam.y + J[7] * lam.z,
                         J[2] * lam.x + J[5] * lam.y + J[8] * lam.z};
            th[0] += fr.s * lam.x;
            th[1] += fr.s * lam.y;
            th[2] += fr.s * lam.z;
            return;
        }
        case TP_FIELD_DIPOLE: {
            // B = K/r^3 (3 (mh.rh) rh - mh), K = coef |m|; the Jacobian is
            // symmetric: J^T l = K/r^4 (3 mh (rh.l) + 3 (mh.rh) l
            //                   + 3 (mh.l) rh - 15 (mh.rh)(rh.l) rh)
            // and dB/dm = coef/r^3 (3 rh rh^T - I)
            F3 d{(p.hi[0] - f.cf[0]) + p.lo[0], (p.hi[1] - f.cf[1]) + p.lo[1], (p.hi[2] - f.cf[2]) + p.lo[2]};
            F3 mh{f.mhatf[0], f.mhatf[1], f.mhatf[2]};
            float ir = __frsqrt_rn(dot(d, d));
            F3 rh = ir * d;
            float mr = dot(mh, rh), rl = dot(rh, lam), ml = dot(mh, lam);
            float k4 = (f.Kf * ir) * ir * ir * ir;
            lx = lx + k4 * ((3.0f * rl) * mh + (3.0f * mr) * lam + (3.0f * ml - 15.0f * mr * rl) * rh);
            double k3 = fr.s * f.coef * (double)ir * (double)ir * (double)ir;
            th[0] += k3 * (3.0 * (double)rl * (double)rh.x - (double)lam.x);
            th[1] += k3 * (3.0 * (double)rl * (double)rh.y - (double)lam.y);
            th[2] += k3 * (3.0 * (double)rl * (double)rh.z - (double)lam.z);
            return;
        }
        default:  // zero / uniform: gradient of a uniform offset
            th[0] += fr.s * lam.x;
            th[1] += fr.s * lam.y;
            th[2] += fr.s * lam.z;
            return;
    }
}

template <int FK>
__device__ __forceinline__ F3 adj_step_gen(const AdjArgs& A, const CPos& p, F3 v, float h, F3 lo, F3& lx,
                                           double* thE, double* thB, Frame& fr) {
    const DevFields& F = A.a.f;
    GridKeep kE, kB;
    kE.ok = kB.ok = true;
    F3 E = (FK == FK_GENERIC && F.E.kind == TP_FIELD_GRID) ? grid_eval_keep(F.E, p, kE)
                                                            : analytic_eval32(F.E, p, A.a.t0);
    F3 B = (FK == FK_GENERIC && F.B.kind == TP_FIELD_GRID) ? grid_eval_keep(F.B, p, kB)
                                                            : analytic_eval32(F.B, p, A.a.t0);
    UAdj u = u_adjoint(v, E, B, h, lo);
    field_adj(F.E, p, kE, u.lE, A.g_E, lx, thE, fr);
    field_adj(F.B, p, kB, u.lB, A.g_B, lx, thB, fr);
    return u.lv;
}

template <int FK>
__device__ __forceinline__ F3 adj_step(const AdjArgs& A, const CPos& p, F3 v, float h, F3 lo, F3& lx,
                                       double* thE, double* thB, Frame& fr) {
    if (FK == FK_EBGRID) return adj_step_eb(A, p, v, h, lo, lx, fr);
    return adj_step_gen<FK>(A, p, v, h, lo, lx, thE, thB, fr);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

}  // namespace

// ------------------------------------------------------------------ kernels
template <int FK>
__global__ void __launch_bounds__(256) k_adj_forward(AdjArgs A) {
    const BorisArgs& a = A.a;
    const double dt = a.dt;
    const float dth = (float)dt, dtl = (float)(dt - (double)dth);
    const float h = vfac<false>(a, dt);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double* u0 = a.u0 + 6 * i;
        CPos p;
        cpos_init(a, p, u0);
        CV v = cv_from(u0 + 3);
        F3 E, B;
        eval_EB32t<FK>(a.f, p, a.t0, E, B);
        v = vel32<false>(v, E, B, a, -0.5 * dt);
        int64_t s = 0, left = 0;
        for (int64_t k = 0; k < A.nt; ++k) {
            if (left == 0) {
                store_ck(A, s, i, p, v);
                ++s;
                left = A.K;
            }
            --left;
            eval_EB32t<FK>(a.f, p, a.t0, E, B);
            v = vel32h<false>(v, E, B, a, h);
            cpos_push_cv(a, p, v, dth, dtl);
        }
        if (A.nt == 0) store_ck(A, 0, i, p, v);
        eval_EB32t<FK>(a.f, p, a.t0, E, B);
        CV vf = vel32<false>(v, E, B, a, A.dt_final);
        double* uo = A.u_final + 6 * i;
        uo[0] = cpos_value(a, p, 0);
        uo[1] = cpos_value(a, p, 1);
        uo[2] = cpos_value(a, p, 2);
        uo[3] = (double)vf.h.x + (double)vf.l.x;
        uo[4] = (double)vf.h.y + (double)vf.l.y;
        uo[5] = (double)vf.h.z + (double)vf.l.z;
    }
}

template <int FK>
__global__ void __launch_bounds__(256) k_adj_backward(AdjArgs A) {
    const BorisArgs& a = A.a;
    const double dt = a.dt;
    const float dtf = (float)dt;
    const float dth = dtf, dtl = (float)(dt - (double)dth);
    const float h = vfac<false>(a, dt);
    const float h_fin = vfac<false>(a, A.dt_final);
    const float h_ini = vfac<false>(a, -0.5 * dt);
    const int G = A.G;
    double thE[3] = {0.0, 0.0, 0.0}, thB[3] = {0.0, 0.0, 0.0};
    int mx = INT_MIN;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        // cotangent of the final save, normalised: lambda = g / 2^e
        const double* gf = A.g_final + 6 * i;
        double gm = fmax(fmax(fmax(fabs(gf[0]), fabs(gf[1])), fmax(fabs(gf[2]), fabs(gf[3]))),
                         fmax(fabs(gf[4]), fabs(gf[5])));
        Frame fr;
        fr.e = (gm > 0.0 && gm <= 1.0e300) ? ilogb(gm) : 0;
        fr.mx = INT_MIN;
        frame_set(fr, G);
        const double is = ldexp(1.0, -fr.e);
        F3 lx{(float)(gf[0] * is), (float)(gf[1] * is), (float)(gf[2] * is)};
        F3 lv{(float)(gf[3] * is), (float)(gf[4] * is), (float)(gf[5] * is)};
        for (int64_t s = A.S - 1; s >= 0; --s) {
            CPos p;
            CV v;
            load_ck(A, s, i, p, v);
            const int64_t k0 = s * A.K;
            const int m = (int)((A.nt - k0 < A.K) ? A.nt - k0 : A.K);
            for (int j = 0; j < m; ++j) {
                store_rec(A, j, i, p, v.h);
                F3 E, B;
                eval_EB32t<FK>(a.f, p, a.t0, E, B);
                v = vel32h<false>(v, E, B, a, h);
                cpos_push_cv(a, p, v, dth, dtl);
            }
            if (s == A.S - 1) {  // final save
                lv = adj_step<FK>(A, p, v.h, h_fin, lv, lx, thE, thB, fr);
                renorm(lx, lv, fr, G);
            }
            if (m > 0) {
                // the record of the next (earlier) step is loaded one step ahead
                CPos q;
                F3 vh;
                load_rec(A, m - 1, i, q, vh);
                for (int j = m - 1; j >= 0; --j) {
                    CPos qn = q;
                    F3 vn = vh;
                    if (j > 0) load_rec(A, j - 1, i, qn, vn);
                    F3 lo = lv + dtf * lx;
                    lv = adj_step<FK>(A, q, vh, h, lo, lx, thE, thB, fr);
                    renorm(lx, lv, fr, G);
                    q = qn;
                    vh = vn;
                }
            }
        }
        // initial half step back
        const double* u0 = a.u0 + 6 * i;
        CPos p0;
        cpos_init(a, p0, u0);
        CV v0 = cv_from(u0 + 3);
        lv = adj_step<FK>(A, p0, v0.h, h_ini, lv, lx, thE, thB, fr);
        double* go = A.g_u0 + 6 * i;
        go[0] = fr.s * lx.x;
        go[1] = fr.s * lx.y;
        go[2] = fr.s * lx.z;
        go[3] = fr.s * lv.x;
        go[4] = fr.s * lv.y;
        go[5] = fr.s * lv.z;
        mx = max(mx, fr.mx);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0 && mx != INT_MIN) atomicMax(A.need, mx);
    if (FK != FK_EBGRID) {
        bool any = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            thE[k] = warp_sum(thE[k]);
            thB[k] = warp_sum(thB[k]);
            any = any || thE[k] != 0.0 || thB[k] != 0.0;
        }
        if ((threadIdx.x & 31) == 0 && any) {
            for (int k = 0; k < 3; ++k) {
                atomicAdd(A.g_param + k, thE[k]);
                atomicAdd(A.g_param + 3 + k, thB[k]);
            }
        }
    }
}

// --------------------------------------------- segmented backward, E/B grid
// For an interleaved E/B grid the backward pass runs as two kernels per
// checkpoint segment.  Recompute reads the field table and streams, for every
// step, the update's inputs and the field's value and Jacobian to the
// records.  Reverse reads the records and accumulates into the gradient
// table.  Each kernel's random-access working set is one 32-byte-per-node
// table, which fits in L2; the records stream through with evict-first hints.
constexpr int kRecEB = 33;  // cell xyz (int; x = -1 outside the grid), fraction xyz, v, E, B, dE/dx.., dB/dx..
constexpr int kRecEB4 = 9;  // as float4 words (3 floats of padding)

// L2 policy for data read once
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// streaming store: no L1 allocation, evict-first in L2
__device__ __forceinline__ void st_once(float4* p, float4 v, uint64_t pol) {
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x),
                 "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}

// field value at p (the forward's arithmetic) with its record for slot j;
// the record is written with streaming (evict-first) stores
__device__ __forceinline__ void record_step_eb(const AdjArgs& A, const CPos& p, F3 v, int j, int64_t i,
                                               uint64_t once, F3& E, F3& B) {
    const DevFields& F = A.a.f;
    const int64_t n = A.a.n;
    float4* r = reinterpret_cast<float4*>(A.rec) + (int64_t)j * kRecEB4 * n + i;
    AxF ax, ay, az;
    if (!axes32(F.B, p, ax, ay, az)) {
        E = nanf3_();
        B = E;
        st_once(r, make_float4(__int_as_float(-1), 0.0f, 0.0f, 0.0f), once);
        return;
    }
    int nd[8];
    tri_nodes(F.B, ax, ay, az, nd);
    float4 e[8], b[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) ldg_node8(F.eb32 + 2 * (int64_t)nd[c], e[c], b[c]);
    st_once(r, make_float4(__int_as_float(ax.i0), __int_as_float(ay.i0), __int_as_float(az.i0), ax.f), once);
    st_once(r + n, make_float4(ay.f, az.f, v.x, v.y), once);
    F3 Ex, Ey, Ez;
    tri_val_jac(e, ax, ay, az, E, Ex, Ey, Ez);
    st_once(r + 2 * n, make_float4(v.z, E.x, E.y, E.z), once);
    F3 Bx, By, Bz;
    tri_val_jac(b, ax, ay, az, B, Bx, By, Bz);
    st_once(r + 3 * n, make_float4(B.x, B.y, B.z, Ex.x), once);
    st_once(r + 4 * n, make_float4(Ex.y, Ex.z, Ey.x, Ey.y), once);
    st_once(r + 5 * n, make_float4(Ey.z, Ez.x, Ez.y, Ez.z), once);
    st_once(r + 6 * n, make_float4(Bx.x, Bx.y, Bx.z, By.x), once);
    st_once(r + 7 * n, make_float4(By.y, By.z, Bz.x, Bz.y), once);
    st_once(r + 8 * n, make_float4(Bz.z, 0.0f, 0.0f, 0.0f), once);
}

// Asynchronous copy of one step's record (kRecEB4 float4 words of particle i)
// into this thread's shared-memory slot, as one cp.async group.
__device__ __forceinline__ void rec_prefetch(const AdjArgs& A, int j, int64_t i, float4* slot, int stride,
                                             uint64_t pol) {
    const int64_t n = A.a.n;
    const float4* r = reinterpret_cast<const float4*>(A.rec) + (int64_t)j * kRecEB4 * n + i;
#pragma unroll
    for (int k = 0; k < kRecEB4; ++k) {
        unsigned d = (unsigned)__cvta_generic_to_shared(slot + k * stride);
        asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(r + k * n),
                     "l"(pol)
                     : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One node-gradient contribution: the cell (x = -1: none), its fractions and
// the frame-scaled cotangents of E and B.
struct Contrib {
    int i0[3];
    float f[3];
    F3 lE, lB;
};

// adjoint of one velocity update from its record (q: kRecEB4 words, `stride`
// apart); returns the cotangent of the input velocity, adds to lx and leaves
// the step's node-gradient contribution in ct
__device__ __forceinline__ F3 reverse_step_eb(const float4* qp, int stride, float h, F3 lo, F3& lx, Frame& fr,
                                              Contrib& ct) {
    float4 q[kRecEB4];
#pragma unroll
    for (int k = 0; k < kRecEB4; ++k) q[k] = qp[k * stride];
    const int ix = __float_as_int(q[0].x);
    ct.i0[0] = -1;
    if (ix < 0) {
        lx = nanf3_();
        return nanf3_();
    }
    F3 v{q[1].z, q[1].w, q[2].x}, E{q[2].y, q[2].z, q[2].w}, B{q[3].x, q[3].y, q[3].z};
    UAdj u = u_adjoint(v, E, B, h, lo);
    lx = lx + jt({q[3].w, q[4].x, q[4].y}, {q[4].z, q[4].w, q[5].x}, {q[5].y, q[5].z, q[5].w}, u.lE) +
         jt({q[6].x, q[6].y, q[6].z}, {q[6].w, q[7].x, q[7].y}, {q[7].z, q[7].w, q[8].x}, u.lB);
    if (fr.f != 0.0f) {
        float m = fmaxf(fmaxf(fmaxf(fabsf(u.lE.x), fabsf(u.lE.y)), fmaxf(fabsf(u.lE.z), fabsf(u.lB.x))),
                        fmaxf(fabsf(u.lB.y), fabsf(u.lB.z)));
        fr.mx = max(fr.mx, fexp(m) + fr.e);
        ct.i0[0] = ix;
        ct.i0[1] = __float_as_int(q[0].y);
        ct.i0[2] = __float_as_int(q[0].z);
        ct.f[0] = q[0].w;
        ct.f[1] = q[1].x;
        ct.f[2] = q[1].y;
        ct.lE = fr.f * u.lE;
        ct.lB = fr.f * u.lB;
    }
    return u.lv;
}

// Warp-transposed scatter of the warp's 32 contributions.  Each lane stages
// its particle's 8 node indices, 8 weights and the two scaled cotangents
// (24 words); then in each of 16 rounds the lanes cover two particles x 8
// corners x (E, B) half, so one reduction instruction touches the nodes of
// two particles (about 16 sectors, the two halves of a node in one 32-byte
// sector) instead of 32 unrelated ones.  All 32 lanes of the warp must call
// it (lanes without a contribution pass i0[0] = -1).
constexpr int kStage = 24;  // staged words per lane: nodes[8], weights[8], lE xyz, pad, lB xyz, pad

__device__ __forceinline__ void scatter_warp_eb(const AdjArgs& A, float* stage, const Contrib& ct, uint64_t pol) {
    const int lane = threadIdx.x & 31;
    const unsigned have = __ballot_sync(0xffffffffu, ct.i0[0] >= 0);
    if (!have) return;  // warp-uniform
    if (ct.i0[0] >= 0) {
        const DevField& g = A.a.f.B;
        AxF ax, ay, az;
        AxF* axs[3] = {&ax, &ay, &az};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            axs[k]->i0 = ct.i0[k];
            axs[k]->i1 = (g.bc == TP_BC_PERIODIC && ct.i0[k] + 1 == g.n[k]) ? 0 : ct.i0[k] + 1;
            axs[k]->f = ct.f[k];
            axs[k]->ds = 0.0f;
        }
        int nd[8];
        float w[8];
        tri_nodes(g, ax, ay, az, nd);
        tri_weights(ax, ay, az, w);
        float4* me = reinterpret_cast<float4*>(stage + lane * kStage);
        me[0] = make_float4(__int_as_float(nd[0]), __int_as_float(nd[1]), __int_as_float(nd[2]), __int_as_float(nd[3]));
        me[1] = make_float4(__int_as_float(nd[4]), __int_as_float(nd[5]), __int_as_float(nd[6]), __int_as_float(nd[7]));
        me[2] = make_float4(w[0], w[1], w[2], w[3]);
        me[3] = make_float4(w[4], w[5], w[6], w[7]);
        me[4] = make_float4(ct.lE.x, ct.lE.y, ct.lE.z, 0.0f);
        me[5] = make_float4(ct.lB.x, ct.lB.y, ct.lB.z, 0.0f);
    }
    __syncwarp();
    const int c = (lane & 15) >> 1, h = lane & 1;
    for (int r = 0; r < 16; ++r) {
        const int src = 2 * r + (lane >> 4);
        if ((have >> src) & 1u) {
            const float* q = stage + src * kStage;
            const int node = __float_as_int(q[c]);
            const float w = q[8 + c];
            const float4 l = *reinterpret_cast<const float4*>(q + 16 + 4 * h);
            red_add3(A.g_eb + 2 * (int64_t)node + h, w * l.x, w * l.y, w * l.z, pol);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ int seg_steps(const AdjArgs& A, int64_t s) {
    const int64_t k0 = s * A.K;
    return (int)((A.nt - k0 < A.K) ? A.nt - k0 : A.K);
}

__global__ void __launch_bounds__(128, 4) k_adj_recompute_eb(AdjArgs A, int64_t s) {
    const BorisArgs& a = A.a;
    const double dt = a.dt;
    const float dth = (float)dt, dtl = (float)(dt - (double)dth);
    const float h = vfac<false>(a, dt);
    const int m = seg_steps(A, s);
    const uint64_t once = l2_evict_first();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        CPos p;
        CV v;
        load_ck(A, s, i, p, v);
        for (int j = 0; j < m; ++j) {
            F3 E, B;
            record_step_eb(A, p, v.h, j, i, once, E, B);
            v = vel32h<false>(v, E, B, a, h);
            cpos_push_cv(a, p, v, dth, dtl);
        }
        if (s == A.S - 1) {  // the final save's update, at (x_N, v_{N-1/2})
            F3 E, B;
            record_step_eb(A, p, v.h, m, i, once, E, B);
        }
    }
}

constexpr int kRevStages = 2;  // records in flight per thread (shared memory ring)

// The particle loop is uniform over the block (lanes past n run empty) so
// that whole warps take part in scatter_warp_eb.
__global__ void __launch_bounds__(128, 4) k_adj_reverse_eb(AdjArgs A, int64_t s) {
    extern __shared__ float4 smem4[];  // ring [kRevStages][kRecEB4][blockDim.x], then staging
    float4* ring = smem4;
    float* stage = reinterpret_cast<float*>(smem4 + kRevStages * kRecEB4 * blockDim.x) +
                   (threadIdx.x & ~31) * kStage;
    const BorisArgs& a = A.a;
    const double dt = a.dt;
    const float dtf = (float)dt;
    const float h = vfac<false>(a, dt);
    const int G = A.G;
    const int m = seg_steps(A, s);
    const int64_t n = a.n;
    const int stride = blockDim.x;
    const uint64_t keep = l2_evict_last();
    const uint64_t once = l2_evict_first();
    int mx = INT_MIN;
    for (int64_t ib = (int64_t)blockIdx.x * blockDim.x; ib < n; ib += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = ib + threadIdx.x;
        const bool live = i < n;
        // records m-1, m-2, ... stream into the ring ahead of their use
#pragma unroll
        for (int d = 0; d < kRevStages; ++d) {
            const int j = m - 1 - d;
            if (live && j >= 0)
                rec_prefetch(A, j, i, ring + (j % kRevStages) * kRecEB4 * stride + threadIdx.x, stride, once);
            cp_async_commit();
        }
        F3 lx{0.0f, 0.0f, 0.0f}, lv{0.0f, 0.0f, 0.0f};
        Frame fr;
        fr.e = 0;
        fr.mx = INT_MIN;
        frame_set(fr, G);
        Contrib ct;
        ct.i0[0] = -1;
        float* st = A.lam + i;
        if (s == A.S - 1) {
            if (live) {
                // cotangent of the final save, normalised: lambda = g / 2^e
                const double* gf = A.g_final + 6 * i;
                double gm = fmax(fmax(fmax(fabs(gf[0]), fabs(gf[1])), fmax(fabs(gf[2]), fabs(gf[3]))),
                                 fmax(fabs(gf[4]), fabs(gf[5])));
                fr.e = (gm > 0.0 && gm <= 1.0e300) ? ilogb(gm) : 0;
                frame_set(fr, G);
                const double is = ldexp(1.0, -fr.e);
                lx = {(float)(gf[0] * is), (float)(gf[1] * is), (float)(gf[2] * is)};
                lv = {(float)(gf[3] * is), (float)(gf[4] * is), (float)(gf[5] * is)};
                // the final save's record (slot m) is read directly
                const float4* r = reinterpret_cast<const float4*>(A.rec) + (int64_t)m * kRecEB4 * n + i;
                lv = reverse_step_eb(r, (int)n, vfac<false>(a, A.dt_final), lv, lx, fr, ct);
                renorm(lx, lv, fr, G);
            }
            scatter_warp_eb(A, stage, ct, keep);
        } else if (live) {
            lx = {st[0], st[n], st[2 * n]};
            lv = {st[3 * n], st[4 * n], st[5 * n]};
            fr.e = __float_as_int(st[6 * n]);
            fr.mx = __float_as_int(st[7 * n]);
            frame_set(fr, G);
        }
        for (int j = m - 1; j >= 0; --j) {
            cp_async_wait<kRevStages - 1>();  // this thread's copy of record j has landed
            ct.i0[0] = -1;
            if (live) {
                F3 lo = lv + dtf * lx;
                lv = reverse_step_eb(ring + (j % kRevStages) * kRecEB4 * stride + threadIdx.x, stride, h, lo, lx, fr,
                                     ct);
                renorm(lx, lv, fr, G);
            }
            // refill the slot just consumed with record j - kRevStages
            const int jn = j - kRevStages;
            if (live && jn >= 0)
                rec_prefetch(A, jn, i, ring + (jn % kRevStages) * kRecEB4 * stride + threadIdx.x, stride, once);
            cp_async_commit();
            scatter_warp_eb(A, stage, ct, keep);
        }
        cp_async_wait<0>();
        if (!live) continue;
        if (s == 0) {
            // initial half step back, v_{-1/2} = U(v_0, x_0, -dt/2)
            const double* u0 = a.u0 + 6 * i;
            CPos p0;
            cpos_init(a, p0, u0);
            CV v0 = cv_from(u0 + 3);
            lv = adj_step_eb(A, p0, v0.h, vfac<false>(a, -0.5 * dt), lv, lx, fr);
            double* go = A.g_u0 + 6 * i;
            go[0] = fr.s * lx.x;
            go[1] = fr.s * lx.y;
            go[2] = fr.s * lx.z;
            go[3] = fr.s * lv.x;
            go[4] = fr.s * lv.y;
            go[5] = fr.s * lv.z;
            mx = max(mx, fr.mx);
        } else {
            st[0] = lx.x;
            st[n] = lx.y;
            st[2 * n] = lx.z;
            st[3 * n] = lv.x;
            st[4 * n] = lv.y;
            st[5 * n] = lv.z;
            st[6 * n] = __int_as_float(fr.e);
            st[7 * n] = __int_as_float(fr.mx);
        }
    }
    if (s == 0) {
        mx = __reduce_max_sync(0xffffffffu, mx);
        if ((threadIdx.x & 31) == 0 && mx != INT_MIN) atomicMax(A.need, mx);
    }
}

// ------------------------------------- fused backward, E/B grid, short segments
// With checkpoint segments of at most kFusedMaxK steps the whole backward
// pass is one kernel.  Each thread walks its particle's segments from last to
// first: it recomputes the segment from its checkpoint into its own records
// in shared memory, then runs them backwards through the adjoint step and
// the warp-transposed scatter.  Records never reach global memory and the
// cotangent stays in registers from the final save to x_0, so per
// particle-step the pass moves the field gather (8 sectors), the node
// reductions (about 8.1 sectors) and 1/K of a 48-byte checkpoint, against
// the two-kernel pass's additional record write and read (4.5 sectors each).
// The records take K x 120 bytes of shared memory per thread, which the SM
// takes from its L1 cache: K = 2 (3 blocks of 128 threads, L1 left at about
// half) is the fastest; at K = 4 the L1 cache shrinks to 28 KB and the pass
// is slower than the two kernels per segment.
//
// Record of one step, 15 float2 words, [slot][word][thread] in shared memory:
//   0: cell x, y (int; x = -1 outside the grid)   1: cell z, fraction x
//   2: fraction y, z   3: vm x, y   4: vm z, B x   5: B y, z
//   6-14: dE/dx, dE/dy, dE/dz, dB/dx, dB/dy, dB/dz (9 + 9 floats in order)
// (vm = v + hE; the adjoint needs no more)
constexpr int kRecF2 = 15;

__device__ __forceinline__ void record_step_f(const DevFields& F, const CPos& p, F3 v, float h, float2* r,
                                              int stride, F3& E, F3& B) {
    AxF ax, ay, az;
    if (!axes32(F.B, p, ax, ay, az)) {
        E = nanf3_();
        B = E;
        r[0] = make_float2(__int_as_float(-1), 0.0f);
        return;
    }
    int nd[8];
    tri_nodes(F.B, ax, ay, az, nd);
    float4 e[8], b[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) ldg_node8(F.eb32 + 2 * (int64_t)nd[c], e[c], b[c]);
    F3 Ex, Ey, Ez, Bx, By, Bz;
    tri_val_jac(e, ax, ay, az, E, Ex, Ey, Ez);
    tri_val_jac(b, ax, ay, az, B, Bx, By, Bz);
    const F3 vm = vminus(v, E, h);
    r[0] = make_float2(__int_as_float(ax.i0), __int_as_float(ay.i0));
    r[stride] = make_float2(__int_as_float(az.i0), ax.f);
    r[2 * stride] = make_float2(ay.f, az.f);
    r[3 * stride] = make_float2(vm.x, vm.y);
    r[4 * stride] = make_float2(vm.z, B.x);
    r[5 * stride] = make_float2(B.y, B.z);
    r[6 * stride] = make_float2(Ex.x, Ex.y);
    r[7 * stride] = make_float2(Ex.z, Ey.x);
    r[8 * stride] = make_float2(Ey.y, Ey.z);
    r[9 * stride] = make_float2(Ez.x, Ez.y);
    r[10 * stride] = make_float2(Ez.z, Bx.x);
    r[11 * stride] = make_float2(Bx.y, Bx.z);
    r[12 * stride] = make_float2(By.x, By.y);
    r[13 * stride] = make_float2(By.z, Bz.x);
    r[14 * stride] = make_float2(Bz.y, Bz.z);
}

// reverse_step_eb for a shared-memory record of record_step_f
__device__ __forceinline__ F3 reverse_step_f(const float2* r, int stride, float h, F3 lo, F3& lx, Frame& fr,
                                             Contrib& ct) {
    ct.i0[0] = -1;
    float2 q[kRecF2];
#pragma unroll
    for (int k = 0; k < kRecF2; ++k) q[k] = r[k * stride];
    const float2 q0 = q[0];
    if (__float_as_int(q0.x) < 0) {
        lx = nanf3_();
        return nanf3_();
    }
    const F3 vm{q[3].x, q[3].y, q[4].x}, B{q[4].y, q[5].x, q[5].y};
    UAdj u = u_adjoint_vm(vm, B, h, lo);
    lx = lx + jt({q[6].x, q[6].y, q[7].x}, {q[7].y, q[8].x, q[8].y}, {q[9].x, q[9].y, q[10].x}, u.lE) +
         jt({q[10].y, q[11].x, q[11].y}, {q[12].x, q[12].y, q[13].x}, {q[13].y, q[14].x, q[14].y}, u.lB);
    if (fr.f != 0.0f) {
        float m = fmaxf(fmaxf(fmaxf(fabsf(u.lE.x), fabsf(u.lE.y)), fmaxf(fabsf(u.lE.z), fabsf(u.lB.x))),
                        fmaxf(fabsf(u.lB.y), fabsf(u.lB.z)));
        fr.mx = max(fr.mx, fexp(m) + fr.e);
        ct.i0[0] = __float_as_int(q0.x);
        ct.i0[1] = __float_as_int(q0.y);
        ct.i0[2] = __float_as_int(q[1].x);
        ct.f[0] = q[1].y;
        ct.f[1] = q[2].x;
        ct.f[2] = q[2].y;
        ct.lE = fr.f * u.lE;
        ct.lB = fr.f * u.lB;
    }
    return u.lv;
}

// The particle loop is uniform over the block (lanes past n run empty, with
// the same segment and step counts) so that whole warps take part in
// scatter_warp_eb.  No block-level synchronisation: each thread reads only
// the records it wrote.
__global__ void __launch_bounds__(128, 3) k_adj_fused_eb(AdjArgs A) {
    extern __shared__ float4 smem4[];  // records [K][kRecF2][blockDim.x] (float2), then staging
    float2* mine = reinterpret_cast<float2*>(smem4) + threadIdx.x;
    const int stride = blockDim.x;
    float* stage = reinterpret_cast<float*>(reinterpret_cast<float2*>(smem4) + (int64_t)A.K * kRecF2 * stride) +
                   (threadIdx.x & ~31) * kStage;
    const BorisArgs& a = A.a;
    const double dt = a.dt;
    const float dtf = (float)dt, dth = dtf, dtl = (float)(dt - (double)dth);
    const float h = vfac<false>(a, dt);
    const int G = A.G;
    const int64_t n = a.n;
    const uint64_t keep = l2_evict_last();
    int mx = INT_MIN;
    for (int64_t ib = (int64_t)blockIdx.x * blockDim.x; ib < n; ib += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = ib + threadIdx.x;
        const bool live = i < n;
        F3 lx{0.0f, 0.0f, 0.0f}, lv{0.0f, 0.0f, 0.0f};
        Frame fr;
        fr.e = 0;
        fr.mx = INT_MIN;
        if (live) {
            // cotangent of the final save, normalised: lambda = g / 2^e
            const double* gf = A.g_final + 6 * i;
            double gm = fmax(fmax(fmax(fabs(gf[0]), fabs(gf[1])), fmax(fabs(gf[2]), fabs(gf[3]))),
                             fmax(fabs(gf[4]), fabs(gf[5])));
            fr.e = (gm > 0.0 && gm <= 1.0e300) ? ilogb(gm) : 0;
            const double is = ldexp(1.0, -fr.e);
            lx = {(float)(gf[0] * is), (float)(gf[1] * is), (float)(gf[2] * is)};
            lv = {(float)(gf[3] * is), (float)(gf[4] * is), (float)(gf[5] * is)};
        }
        frame_set(fr, G);
        for (int64_t s = A.S - 1; s >= 0; --s) {
            const int m = seg_steps(A, s);
            if (live) {
                CPos p;
                CV v;
                load_ck(A, s, i, p, v);
                for (int j = 0; j < m; ++j) {
                    F3 E, B;
                    record_step_f(a.f, p, v.h, h, mine + j * kRecF2 * stride, stride, E, B);
                    v = vel32h<false>(v, E, B, a, h);
                    cpos_push_cv(a, p, v, dth, dtl);
                }
                if (s == A.S - 1) {  // the final save's update, at (x_N, v_{N-1/2})
                    lv = adj_step_eb(A, p, v.h, vfac<false>(a, A.dt_final), lv, lx, fr);
                    renorm(lx, lv, fr, G);
                }
            }
            for (int j = m - 1; j >= 0; --j) {
                Contrib ct;
                ct.i0[0] = -1;
                if (live) {
                    F3 lo = lv + dtf * lx;
                    lv = reverse_step_f(mine + j * kRecF2 * stride, stride, h, lo, lx, fr, ct);
                    renorm(lx, lv, fr, G);
                }
                scatter_warp_eb(A, stage, ct, keep);
            }
        }
        if (!live) continue;
        // initial half step back, v_{-1/2} = U(v_0, x_0, -dt/2)
        const double* u0 = a.u0 + 6 * i;
        CPos p0;
        cpos_init(a, p0, u0);
        CV v0 = cv_from(u0 + 3);
        lv = adj_step_eb(A, p0, v0.h, vfac<false>(a, -0.5 * dt), lv, lx, fr);
        double* go = A.g_u0 + 6 * i;
        go[0] = fr.s * lx.x;
        go[1] = fr.s * lx.y;
        go[2] = fr.s * lx.z;
        go[3] = fr.s * lv.x;
        go[4] = fr.s * lv.y;
        go[5] = fr.s * lv.z;
        mx = max(mx, fr.mx);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0 && mx != INT_MIN) atomicMax(A.need, mx);
}

// sum of a node-gradient table (stored scaled by 2^-G) into out[0..2]
__global__ void k_table_sum(const float4* tab, int64_t nodes, int stride, int off, int G, double* out) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nodes;
         k += (int64_t)gridDim.x * blockDim.x) {
        float4 q = tab[k * stride + off];
        sx += q.x;
        sy += q.y;
        sz += q.z;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    sz = warp_sum(sz);
    __shared__ double part[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        part[0][wid] = sx;
        part[1][wid] = sy;
        part[2][wid] = sz;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, ldexp(t, G));
    }
}

__global__ void k_table_unpack(const float4* tab, int64_t nodes, int stride, int off, int G, double* out) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    float4 q = tab[k * stride + off];
    out[3 * k + 0] = ldexp((double)q.x, G);
    out[3 * k + 1] = ldexp((double)q.y, G);
    out[3 * k + 2] = ldexp((double)q.z, G);
}

// ---------------------------------------------------------------- launchers
int adjoint_field_config(const DevFields& f) {
    if (f.eb32) return FK_EBGRID;
    if (f.E.kind != TP_FIELD_GRID && f.B.kind != TP_FIELD_GRID) return FK_ANALYTIC;
    return FK_GENERIC;
}

cudaError_t launch_adjoint_forward(const AdjArgs& a, int fk, const LaunchCfg& c, cudaStream_t s) {
    const void* k = fk == FK_EBGRID    ? (const void*)k_adj_forward<FK_EBGRID>
                    : fk == FK_ANALYTIC ? (const void*)k_adj_forward<FK_ANALYTIC>
                                        : (const void*)k_adj_forward<FK_GENERIC>;
    void* args[] = {const_cast<AdjArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(c.grid), dim3(c.block), args, 0, s);
}

// shared memory of k_adj_fused_eb for a block of `block` threads
size_t fused_smem(int64_t K, int block) {
    return (size_t)K * kRecF2 * block * sizeof(float2) + (size_t)kStage * block * sizeof(float);
}

cudaError_t launch_adjoint_backward(const AdjArgs& a, int fk, const LaunchCfg& c, cudaStream_t s) {
    if (fk == FK_EBGRID && adjoint_fused(fk, a.K)) {  // one kernel for the whole pass
        const int block = c.block < 128 ? (c.block < 32 ? 32 : c.block & ~31) : 128;
        const size_t smem = fused_smem(a.K, block);
        cudaError_t e = cudaFuncSetAttribute(k_adj_fused_eb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int64_t g = (a.a.n + block - 1) / block;
        k_adj_fused_eb<<<(unsigned)(g < 0x7fffffff ? g : 0x7fffffff), block, smem, s>>>(a);
        return cudaGetLastError();
    }
    if (fk == FK_EBGRID) {  // two kernels per segment, last segment first
        const size_t smem = (size_t)kRevStages * kRecEB4 * c.block * sizeof(float4) +
                            (size_t)kStage * c.block * sizeof(float);
        cudaError_t e = cudaFuncSetAttribute(k_adj_reverse_eb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        for (int64_t seg = a.S - 1; seg >= 0; --seg) {
            k_adj_recompute_eb<<<c.grid, c.block, 0, s>>>(a, seg);
            k_adj_reverse_eb<<<c.grid, c.block, smem, s>>>(a, seg);
        }
        return cudaGetLastError();
    }
    const void* k = fk == FK_ANALYTIC ? (const void*)k_adj_backward<FK_ANALYTIC>
                                      : (const void*)k_adj_backward<FK_GENERIC>;
    void* args[] = {const_cast<AdjArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(c.grid), dim3(c.block), args, 0, s);
}

// float words of the per-step records of one segment and of the cotangent
// state kept between segments
int64_t adjoint_record_words(int fk, int64_t K, int64_t n) {
    if (adjoint_fused(fk, K)) return 0;
    return fk == FK_EBGRID ? (K + 1) * kRecEB4 * 4 * n : K * kRec * n;
}
int64_t adjoint_state_words(int fk, int64_t K, int64_t n) {
    return fk == FK_EBGRID && !adjoint_fused(fk, K) ? 8 * n : 0;
}
bool adjoint_fused(int fk, int64_t K) { return fk == FK_EBGRID && K <= kFusedMaxK; }

cudaError_t launch_table_sum(const float4* tab, int64_t nodes, int stride, int off, int G, double* out,
                             cudaStream_t s) {
    if (nodes <= 0) return cudaSuccess;
    const int block = 256;
    int64_t g = (nodes + block - 1) / block;
    if (g > 148 * 8) g = 148 * 8;
    k_table_sum<<<(unsigned)g, block, 0, s>>>(tab, nodes, stride, off, G, out);
    return cudaGetLastError();
}

cudaError_t launch_table_unpack(const float4* tab, int64_t nodes, int stride, int off, int G, double* out,
                                cudaStream_t s) {
    if (nodes <= 0) return cudaSuccess;
    const int block = 256;
    k_table_unpack<<<(unsigned)((nodes + block - 1) / block), block, 0, s>>>(tab, nodes, stride, off, G, out);
    return cudaGetLastError();
}

}  // namespace tpb
