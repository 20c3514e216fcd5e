// grid_general.cuh -- gridded fields off the trilinear uniform-Cartesian fast
// path: interpolation order 0 / 1 / 3, rectilinear (non-uniform) axes,
// spherical grids and 1-D / 2-D interpolants, in float64.
//
// The reference builds these with build_interpolator
// (src/utility/interpolation.jl:119-311) over FastInterpolations.jl
// (constant_interp, linear_interp, cardinal_interp) and wraps spherical
// grids in SphericalFieldInterpolator (:97-117), which converts the point
// with cart2sph and the interpolated (v_r, v_theta, v_phi) with sph2cartvec
// (src/utility/utility.jl:63-89).
//
// Every function is templated on the scalar S: double for values, Dual3 for
// values with the three partial derivatives d/dx, d/dy, d/dz -- the role
// ForwardDiff plays for the reference's Jacobians (_get_B_jacobian,
// src/utility/utility.jl:386-392).  The value part of a Dual3 evaluation
// performs exactly the double operations, so the two agree bit for bit.
//
// Per axis (u = (x - origin) / spacing on uniform axes):
//   CONSTANT  the nearest node, floor(u + 1/2) (ties to the upper node)
//   LINEAR    cell i = min(floor(u), n - 2), f = u - i; lerp a + f (b - a)
//   CUBIC     the same cell; cubic Hermite with Catmull-Rom slopes
//             m_i = (f_{i+1} - f_{i-1}) / 2 (index units); in the first and
//             last cell of a non-periodic axis the end slope is the
//             three-point one-sided difference (-3 f_0 + 4 f_1 - f_2) / 2
//             (mirrored at the upper end); an axis of two nodes uses the
//             secant slope at both ends.
//   boundaries: FILL_NAN (outside -> NaN), CLAMP (the coordinate clamped,
//   zero derivative outside), PERIODIC (period n nodes) and
//   PERIODIC_INCLUSIVE (period n - 1 nodes; node n - 1 repeats node 0).
//   Non-uniform axes: the cell from a binary search, f = (x - c_i) /
//   (c_{i+1} - c_i); nearest node by distance (ties to the upper node).
// Nodes are combined axis by axis (x innermost, then y, then z): nested lerps
// for LINEAR, ((w0 v0 + w1 v1) + w2 v2) + w3 v3 for CUBIC.
#pragma once

#include "tp_device.cuh"

namespace tpb {

// ---------------------------------------------------------------- Dual3
struct Dual3 {
    double v;
    double d[3];
};

__device__ __forceinline__ double gval(double a) { return a; }
__device__ __forceinline__ double gval(const Dual3& a) { return a.v; }

template <class S>
__device__ __forceinline__ S gconst(double c);
template <>
__device__ __forceinline__ double gconst<double>(double c) { return c; }
template <>
__device__ __forceinline__ Dual3 gconst<Dual3>(double c) { return {c, {0.0, 0.0, 0.0}}; }

__device__ __forceinline__ Dual3 operator+(const Dual3& a, const Dual3& b) {
    return {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}};
}
__device__ __forceinline__ Dual3 operator-(const Dual3& a, const Dual3& b) {
    return {a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}};
}
__device__ __forceinline__ Dual3 operator*(const Dual3& a, const Dual3& b) {
    return {a.v * b.v,
            {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
__device__ __forceinline__ Dual3 operator/(const Dual3& a, const Dual3& b) {
    double q = a.v / b.v;
    return {q, {(a.d[0] - q * b.d[0]) / b.v, (a.d[1] - q * b.d[1]) / b.v, (a.d[2] - q * b.d[2]) / b.v}};
}
__device__ __forceinline__ Dual3 operator+(const Dual3& a, double c) { return {a.v + c, {a.d[0], a.d[1], a.d[2]}}; }
__device__ __forceinline__ Dual3 operator+(double c, const Dual3& a) { return {c + a.v, {a.d[0], a.d[1], a.d[2]}}; }
__device__ __forceinline__ Dual3 operator-(const Dual3& a, double c) { return {a.v - c, {a.d[0], a.d[1], a.d[2]}}; }
__device__ __forceinline__ Dual3 operator-(double c, const Dual3& a) {
    return {c - a.v, {-a.d[0], -a.d[1], -a.d[2]}};
}
__device__ __forceinline__ Dual3 operator*(const Dual3& a, double c) {
    return {a.v * c, {a.d[0] * c, a.d[1] * c, a.d[2] * c}};
}
__device__ __forceinline__ Dual3 operator*(double c, const Dual3& a) {
    return {c * a.v, {c * a.d[0], c * a.d[1], c * a.d[2]}};
}
__device__ __forceinline__ Dual3 operator/(const Dual3& a, double c) {
    return {a.v / c, {a.d[0] / c, a.d[1] / c, a.d[2] / c}};
}

__device__ __forceinline__ double gsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ Dual3 gsqrt(const Dual3& a) {
    double s = sqrt(a.v);
    double k = 0.5 / s;
    return {s, {a.d[0] * k, a.d[1] * k, a.d[2] * k}};
}
__device__ __forceinline__ double gacos(double a) { return acos(a); }
__device__ __forceinline__ Dual3 gacos(const Dual3& a) {
    double k = -1.0 / sqrt(1.0 - a.v * a.v);
    return {acos(a.v), {a.d[0] * k, a.d[1] * k, a.d[2] * k}};
}
__device__ __forceinline__ double gatan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ Dual3 gatan2(const Dual3& y, const Dual3& x) {
    double den = x.v * x.v + y.v * y.v;
    Dual3 o;
    o.v = atan2(y.v, x.v);
    for (int k = 0; k < 3; ++k) o.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
    return o;
}
__device__ __forceinline__ void gsincos(double a, double& s, double& c) { sincos(a, &s, &c); }
__device__ __forceinline__ void gsincos(const Dual3& a, Dual3& s, Dual3& c) {
    double sv, cv;
    sincos(a.v, &sv, &cv);
    s = {sv, {a.d[0] * cv, a.d[1] * cv, a.d[2] * cv}};
    c = {cv, {-(a.d[0] * sv), -(a.d[1] * sv), -(a.d[2] * sv)}};
}

// ---------------------------------------------------------------- axes
template <class S>
struct GAx {
    int32_t i[4];
    S w[4];      // LINEAR: w[0] = fraction; CUBIC: node weights
    int32_t k;   // nodes along the axis (1 .. 4)
};

__device__ __forceinline__ int64_t gwrap(int64_t i, int64_t m) {
    int64_t r = i % m;
    return r < 0 ? r + m : r;
}

// Cubic Hermite basis at t and the node weights of the cell (see header).
template <class S>
__device__ __forceinline__ void cubic_weights(const S& t, int64_t i, int64_t na, bool periodic, int64_t m,
                                              GAx<S>& o) {
    S t2 = t * t;
    S t3 = t2 * t;
    S h00 = (2.0 * t3 - 3.0 * t2) + 1.0;
    S h10 = (t3 - 2.0 * t2) + t;
    S h01 = 3.0 * t2 - 2.0 * t3;
    S h11 = t3 - t2;
    if (periodic) {
        o.k = 4;
        for (int q = 0; q < 4; ++q) o.i[q] = (int32_t)gwrap(i - 1 + q, m);
        o.w[0] = -0.5 * h10;
        o.w[1] = h00 - 0.5 * h11;
        o.w[2] = h01 + 0.5 * h10;
        o.w[3] = 0.5 * h11;
        return;
    }
    if (na == 2) {
        o.k = 2;
        o.i[0] = 0;
        o.i[1] = 1;
        o.w[0] = (h00 - h10) - h11;
        o.w[1] = (h01 + h10) + h11;
        return;
    }
    if (i == 0) {
        o.k = 3;
        o.i[0] = 0;
        o.i[1] = 1;
        o.i[2] = 2;
        o.w[0] = (h00 - 1.5 * h10) - 0.5 * h11;
        o.w[1] = h01 + 2.0 * h10;
        o.w[2] = 0.5 * h11 - 0.5 * h10;
        return;
    }
    if (i == na - 2) {
        o.k = 3;
        o.i[0] = (int32_t)(na - 3);
        o.i[1] = (int32_t)(na - 2);
        o.i[2] = (int32_t)(na - 1);
        o.w[0] = 0.5 * h11 - 0.5 * h10;
        o.w[1] = h00 - 2.0 * h11;
        o.w[2] = (h01 + 0.5 * h10) + 1.5 * h11;
        return;
    }
    o.k = 4;
    for (int q = 0; q < 4; ++q) o.i[q] = (int32_t)(i - 1 + q);
    o.w[0] = -0.5 * h10;
    o.w[1] = h00 - 0.5 * h11;
    o.w[2] = h01 + 0.5 * h10;
    o.w[3] = 0.5 * h11;
}

// Axis a of a general grid at coordinate x; false where the field is NaN.
template <class S>
__device__ __forceinline__ bool gaxis(const DevField& g, int a, S x, GAx<S>& o) {
    const int64_t na = g.n[a];
    if (na == 1) {  // unused axis of a 1-D / 2-D interpolant
        o.k = 1;
        o.i[0] = 0;
        return true;
    }
    const int bc = g.abc[a];
    const double* c = g.ax[a];
    if (c) {  // non-uniform axis: LINEAR or CONSTANT, FILL_NAN or CLAMP
        const double lo = __ldg(c), hi = __ldg(c + na - 1);
        double xv = gval(x);
        if (bc == TP_BC_CLAMP) {
            if (xv < lo) x = gconst<S>(lo);
            else if (xv > hi) x = gconst<S>(hi);
            xv = gval(x);
        } else if (!(xv >= lo && xv <= hi)) {
            return false;
        }
        int64_t il = 0, ih = na - 1;
        while (ih - il > 1) {
            int64_t mid = (il + ih) >> 1;
            if (__ldg(c + mid) <= xv) il = mid;
            else ih = mid;
        }
        const double cl = __ldg(c + il), ch = __ldg(c + il + 1);
        if (g.order == TP_ORDER_CONSTANT) {
            o.k = 1;
            o.i[0] = (int32_t)((xv - cl < ch - xv) ? il : il + 1);
            return true;
        }
        o.k = 2;
        o.i[0] = (int32_t)il;
        o.i[1] = (int32_t)(il + 1);
        o.w[0] = (x - cl) / (ch - cl);
        return true;
    }
    S u = (x - g.x0[a]) * g.inv_dx[a];
    const bool periodic = bc == TP_BC_PERIODIC || bc == TP_BC_PERIODIC_INCLUSIVE;
    const int64_t m = bc == TP_BC_PERIODIC ? na : na - 1;  // period in nodes
    const double umax = (double)(na - 1);
    if (g.order == TP_ORDER_CONSTANT) {
        double uv = gval(u);
        int64_t i;
        if (periodic) {
            i = gwrap((int64_t)floor(uv + 0.5), m);
        } else {
            if (bc == TP_BC_CLAMP) uv = uv < 0.0 ? 0.0 : (uv > umax ? umax : uv);
            else if (!(uv >= 0.0 && uv <= umax)) return false;
            i = (int64_t)floor(uv + 0.5);
        }
        o.k = 1;
        o.i[0] = (int32_t)i;
        return true;
    }
    int64_t i;
    S f;
    if (periodic) {
        double fl = floor(gval(u));
        f = u - fl;
        i = gwrap((int64_t)fl, m);
    } else {
        double uv = gval(u);
        if (bc == TP_BC_CLAMP) {
            if (uv < 0.0) u = gconst<S>(0.0);
            else if (uv > umax) u = gconst<S>(umax);
        } else if (!(uv >= 0.0 && uv <= umax)) {
            return false;
        }
        i = (int64_t)floor(gval(u));
        if (i > na - 2) i = na - 2;
        f = u - (double)i;
    }
    if (g.order == TP_ORDER_CUBIC) {
        cubic_weights(f, i, na, periodic, m, o);
        return true;
    }
    o.k = 2;
    o.i[0] = (int32_t)i;
    o.i[1] = (int32_t)((bc == TP_BC_PERIODIC && i + 1 == na) ? 0 : i + 1);
    o.w[0] = f;
    return true;
}

// one node (3 components) of the per-node table as doubles; T32 reads the
// float table (the FP32C kernels' copy, half the bytes of a float64 table)
template <bool T32>
__device__ __forceinline__ void gnode(const DevField& g, int64_t idx, double v[3]) {
    if (T32) {
        float4 q = __ldg(g.tab32 + idx);
        v[0] = (double)q.x;
        v[1] = (double)q.y;
        v[2] = (double)q.z;
    } else if (g.f64) {
        const double2* p = reinterpret_cast<const double2*>(g.tab) + 2 * idx;
        double2 a = __ldg(p), b = __ldg(p + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
    } else {
        float4 q = __ldg(reinterpret_cast<const float4*>(g.tab) + idx);
        v[0] = (double)q.x;
        v[1] = (double)q.y;
        v[2] = (double)q.z;
    }
}

// combine the values along one axis
template <class S, class V>
__device__ __forceinline__ S gcombine(const GAx<S>& a, bool linear, const V* v) {
    if (a.k == 1) return gconst<S>(0.0) + v[0];
    if (linear) return v[0] + a.w[0] * (v[1] - v[0]);
    S acc = a.w[0] * v[0] + a.w[1] * v[1];
    for (int q = 2; q < a.k; ++q) acc = acc + a.w[q] * v[q];
    return acc;
}

// Value-only interpolation when every axis of the cell takes the same
// number of nodes: 64 nodes of an interior cubic cell, 8 of a linear cell, 1
// nearest node.  Unrolled with the partial sums accumulated as the nodes
// arrive, so nothing is indexed at run time and the sums stay in registers;
// the operations and their order are those of the general loop below.
template <bool T32>
__device__ __forceinline__ void ginterp_cubic4(const DevField& g, const GAx<double> A[3], double out[3]) {
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    double oz[3];
#pragma unroll
    for (int kz = 0; kz < 4; ++kz) {
        double oy[3];
#pragma unroll
        for (int ky = 0; ky < 4; ++ky) {
            const int64_t base = (int64_t)A[1].i[ky] * nx + (int64_t)A[2].i[kz] * nxy;
            double ox[3];
#pragma unroll
            for (int kx = 0; kx < 4; ++kx) {
                double v[3];
                gnode<T32>(g, base + A[0].i[kx], v);
#pragma unroll
                for (int c = 0; c < 3; ++c) ox[c] = kx == 0 ? A[0].w[0] * v[c] : ox[c] + A[0].w[kx] * v[c];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) oy[c] = ky == 0 ? A[1].w[0] * ox[c] : oy[c] + A[1].w[ky] * ox[c];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) oz[c] = kz == 0 ? A[2].w[0] * oy[c] : oz[c] + A[2].w[kz] * oy[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = oz[c];
}

template <bool T32>
__device__ __forceinline__ void ginterp_linear2(const DevField& g, const GAx<double> A[3], double out[3]) {
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    double cz[2][3];
#pragma unroll
    for (int kz = 0; kz < 2; ++kz) {
        double cy[2][3];
#pragma unroll
        for (int ky = 0; ky < 2; ++ky) {
            const int64_t base = (int64_t)A[1].i[ky] * nx + (int64_t)A[2].i[kz] * nxy;
            double v0[3], v1[3];
            gnode<T32>(g, base + A[0].i[0], v0);
            gnode<T32>(g, base + A[0].i[1], v1);
#pragma unroll
            for (int c = 0; c < 3; ++c) cy[ky][c] = v0[c] + A[0].w[0] * (v1[c] - v0[c]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) cz[kz][c] = cy[0][c] + A[1].w[0] * (cy[1][c] - cy[0][c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = cz[0][c] + A[2].w[0] * (cz[1][c] - cz[0][c]);
}

template <bool T32>
__device__ __forceinline__ bool ginterp_fixed(const DevField&, const GAx<Dual3>*, bool, Dual3*) {
    return false;
}
template <bool T32>
__device__ __forceinline__ bool ginterp_fixed(const DevField& g, const GAx<double>* A, bool lin, double* out) {
    const int k = A[0].k;
    if (A[1].k != k || A[2].k != k) return false;
    if (k == 4) {
        ginterp_cubic4<T32>(g, A, out);
        return true;
    }
    if (k == 2 && lin) {
        ginterp_linear2<T32>(g, A, out);
        return true;
    }
    if (k == 1) {
        double v[3];
        gnode<T32>(g, (int64_t)A[0].i[0] + (int64_t)A[1].i[0] * g.n[0] + (int64_t)A[2].i[0] * ((int64_t)g.n[0] * g.n[1]),
              v);
        for (int c = 0; c < 3; ++c) out[c] = 0.0 + (0.0 + (0.0 + v[c]));
        return true;
    }
    return false;
}

// interpolate the three components at grid coordinates (q0, q1, q2)
template <class S, bool T32>
__device__ __forceinline__ bool ginterp(const DevField& g, const S q[3], S out[3]) {
    GAx<S> A[3];
    bool ok = gaxis(g, 0, q[0], A[0]);
    ok = gaxis(g, 1, q[1], A[1]) && ok;
    ok = gaxis(g, 2, q[2], A[2]) && ok;
    if (!ok) return false;
    const bool lin = g.order == TP_ORDER_LINEAR;
    if (ginterp_fixed<T32>(g, A, lin, out)) return true;
    const int64_t nx = g.n[0], nxy = (int64_t)g.n[0] * g.n[1];
    S cz[4][3];
    for (int kz = 0; kz < A[2].k; ++kz) {
        S cy[4][3];
        for (int ky = 0; ky < A[1].k; ++ky) {
            double vx[4][3];
            const int64_t base = (int64_t)A[1].i[ky] * nx + (int64_t)A[2].i[kz] * nxy;
            for (int kx = 0; kx < A[0].k; ++kx) gnode<T32>(g, base + A[0].i[kx], vx[kx]);
            for (int c = 0; c < 3; ++c) {
                double col[4];
                for (int kx = 0; kx < A[0].k; ++kx) col[kx] = vx[kx][c];
                cy[ky][c] = gcombine<S, double>(A[0], lin, col);
            }
        }
        for (int c = 0; c < 3; ++c) {
            S col[4];
            for (int ky = 0; ky < A[1].k; ++ky) col[ky] = cy[ky][c];
            cz[kz][c] = gcombine<S, S>(A[1], lin, col);
        }
    }
    for (int c = 0; c < 3; ++c) {
        S col[4];
        for (int kz = 0; kz < A[2].k; ++kz) col[kz] = cz[kz][c];
        out[c] = gcombine<S, S>(A[2], lin, col);
    }
    return true;
}

// Field value (and, for S = Dual3, its partial derivatives) at the
// Cartesian point r; false where the field is NaN.  T32: node values from
// the float table.
template <class S, bool T32 = false>
__device__ __forceinline__ bool grid_general_eval(const DevField& g, const S r[3], S out[3]) {
    if (g.geom == TP_GRID_SPHERICAL || g.geom == TP_GRID_SPHERICAL_SCALAR) {
        // cart2sph (src/utility/utility.jl:63-71)
        S rr = gsqrt((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]);
        S q[3];
        if (gval(rr) == 0.0) {
            q[0] = q[1] = q[2] = gconst<S>(0.0);
        } else {
            q[0] = rr;
            q[1] = gacos(r[2] / rr);
            S ph = gatan2(r[1], r[0]);
            if (gval(ph) < 0.0) ph = ph + 6.283185307179586;  // mod2pi
            q[2] = ph;
        }
        S v[3];
        if (!ginterp<S, T32>(g, q, v)) return false;
        if (g.geom == TP_GRID_SPHERICAL_SCALAR) {
            out[0] = v[0];
            out[1] = v[1];
            out[2] = v[2];
            return true;
        }
        // sph2cartvec (src/utility/utility.jl:82-89)
        S st, ct, sp, cp;
        gsincos(q[1], st, ct);
        gsincos(q[2], sp, cp);
        out[0] = ((st * cp) * v[0] + (ct * cp) * v[1]) - sp * v[2];
        out[1] = ((st * sp) * v[0] + (ct * sp) * v[1]) + cp * v[2];
        out[2] = ct * v[0] - st * v[1];
        return true;
    }
    S q[3];
    if (g.ndim == 1) {
        q[0] = r[g.dir];
        q[1] = q[2] = gconst<S>(0.0);
    } else {
        q[0] = r[0];
        q[1] = r[1];
        q[2] = r[2];
    }
    return ginterp<S, T32>(g, q, out);
}

}  // namespace tpb
