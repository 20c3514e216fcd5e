// tp_oracle.hpp -- CPU restatement of TestParticle.jl's particle-push hot path.
//
// TEST INFRASTRUCTURE ONLY.  This header is the parity oracle: the tests, the
// smoke check and the CPU-baseline leg of the benchmark link it (through
// liboracle.so) to check and to time the CUDA library against it.  The
// product library never includes, links or calls it.
//
// Scope (reference = TestParticle.jl v0.23.2, paths relative to its root):
//   boris_velocity_update      src/boris/boris.jl:19-31
//   update_velocity            src/boris/boris.jl:38-45
//   update_velocity_multistep  src/boris/multistep_boris.jl:65-142
//   _prepare_checks / nout     src/boris/boris.jl:345-403
//   _boris_loop! / _boris_single  src/boris/boris.jl:445-557
//   _adaptive_boris_single     src/boris/adaptive_boris.jl:145-266
//   get_B_parameters           src/equations.jl:239-247
//   get_gc_derivatives         src/equations.jl:329-360
//   update_rk4 / _rk4!         src/gc/rk4_gc.jl:7-130
//   update_dp5 / _rk45!        src/gc/rk45_gc.jl:7-173
//   _prepare_gc                src/gc/gc_solver.jl:187-231
//   _get_gc_parameters         src/gc/gc.jl:13-39
//   get_perp_vector            src/utility/utility.jl:119-126
//   fields: ZeroField (src/utility/zero.jl:66-73), trilinear FieldInterpolator
//           (src/utility/interpolation.jl:21-27,217-235; the arithmetic of the
//           third-party FastInterpolations.jl 0.4.11 linear_interp is restated
//           from its published definition, see GridField below).
//
// Floating point.  Compile with -ffp-contract=off.  Julia evaluates these
// expressions without contraction except where `@muladd` (or `@fastmath`)
// rewrites a scalar `a*b + c`; those places call std::fma explicitly and say
// so.  SVector arithmetic under `@muladd` is not fused (the generic muladd
// fallback computes x*y + z), so vector updates are plain multiply-then-add.
// The library's FP64 kernels follow the same order, which makes the two
// bit-identical wherever only +, -, *, /, sqrt and fma are involved.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>

#include "../include/tp_abi.h"

namespace orc {

// ---------------------------------------------------------------- vectors
template <class T>
struct V3 {
    T x, y, z;
};

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
// StaticArrays cross: (a2 b3 - a3 b2, a3 b1 - a1 b3, a1 b2 - a2 b1)
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// StaticArrays dot / sum(abs2, .): ((a1 b1 + a2 b2) + a3 b3)
template <class T> inline T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> inline T abs2sum(V3<T> a) { return (a.x * a.x + a.y * a.y) + a.z * a.z; }
inline double norm(V3<double> a) { return std::sqrt(abs2sum(a)); }

using V3d = V3<double>;

// 3x3 matrix, row-major: J[i][j] = d F_i / d x_j
struct M3 {
    double a[9];
    double operator()(int i, int j) const { return a[3 * i + j]; }
};

// ---------------------------------------------------------------- fields
// Every field offers eval(r, t) and jac(r, t, B, J) (value and Jacobian, the
// role ForwardDiff.jacobian plays in _get_B_jacobian, src/utility/utility.jl:386-392).

struct Field {
    virtual ~Field() {}
    virtual V3d eval(V3d r, double t) const = 0;
    virtual void jac(V3d r, double t, V3d& F, M3& J) const = 0;
    // dF/dt (derivative_t, src/prepare.jl:64-74): zero for static fields
    virtual V3d dtime(V3d, double) const { return {0.0, 0.0, 0.0}; }
};

struct ZeroField : Field {
    V3d eval(V3d, double) const override { return {0.0, 0.0, 0.0}; }
    void jac(V3d, double, V3d& F, M3& J) const override {
        F = {0.0, 0.0, 0.0};
        for (double& v : J.a) v = 0.0;
    }
};

struct UniformField : Field {
    V3d v;
    explicit UniformField(V3d v_) : v(v_) {}
    V3d eval(V3d, double) const override { return v; }
    void jac(V3d, double, V3d& F, M3& J) const override {
        F = v;
        for (double& a : J.a) a = 0.0;
    }
};

// F(x,t) = F0 + J x + rate t, evaluated as ((F0_i + ((J_i0 x + J_i1 y) + J_i2 z)) + rate_i t)
struct AffineField : Field {
    V3d f0;
    M3 Jm;
    V3d rate;
    V3d eval(V3d r, double t) const override {
        V3d F;
        F.x = (f0.x + ((Jm(0, 0) * r.x + Jm(0, 1) * r.y) + Jm(0, 2) * r.z)) + rate.x * t;
        F.y = (f0.y + ((Jm(1, 0) * r.x + Jm(1, 1) * r.y) + Jm(1, 2) * r.z)) + rate.y * t;
        F.z = (f0.z + ((Jm(2, 0) * r.x + Jm(2, 1) * r.y) + Jm(2, 2) * r.z)) + rate.z * t;
        return F;
    }
    void jac(V3d r, double t, V3d& F, M3& J) const override {
        F = eval(r, t);
        J = Jm;
    }
    V3d dtime(V3d, double) const override { return rate; }
};

// Quadratic field F_i = value_i + sum_j J_ij x_j + sum_jk Q_ijk x_j x_k + rate_i t,
// evaluated as ((v_i + ((J_i0 x + J_i1 y) + J_i2 z)) + q_i) + rate_i t with
// q_i = (x (Q_i0.x) + y (Q_i1.x)) + z (Q_i2.x); the reference's quadratic
// test fields (the magnetic bottle of test/test_hybrid.jl:61-68).
struct QuadraticField : Field {
    double v[3], J[9], Q[27], rate[3];
    V3d eval(V3d r, double t) const override {
        double x = r.x, y = r.y, z = r.z, o[3];
        for (int i = 0; i < 3; ++i) {
            const double* Ji = J + 3 * i;
            const double* Qi = Q + 9 * i;
            double lin = (Ji[0] * x + Ji[1] * y) + Ji[2] * z;
            double qx = (Qi[0] * x + Qi[1] * y) + Qi[2] * z;
            double qy = (Qi[3] * x + Qi[4] * y) + Qi[5] * z;
            double qz = (Qi[6] * x + Qi[7] * y) + Qi[8] * z;
            double q = (x * qx + y * qy) + z * qz;
            o[i] = ((v[i] + lin) + q) + rate[i] * t;
        }
        return {o[0], o[1], o[2]};
    }
    void jac(V3d r, double t, V3d& F, M3& Jm) const override {
        F = eval(r, t);
        double x[3] = {r.x, r.y, r.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double* Qi = Q + 9 * i;
                double acc = J[3 * i + j];
                for (int k = 0; k < 3; ++k) acc = acc + (Qi[3 * j + k] + Qi[3 * k + j]) * x[k];
                Jm.a[3 * i + j] = acc;
            }
    }
    V3d dtime(V3d, double) const override { return {rate[0], rate[1], rate[2]}; }
};

// Point dipole B(x) = coef (3 (m.rhat) rhat - m) / d^3, d = |x - c|, evaluated
// in the order of the textbook expression coef * (3*(m.rhat)*rhat - m) / d^3.
struct DipoleField : Field {
    V3d m, c;
    double coef;
    V3d eval(V3d r, double) const override {
        V3d d = r - c;
        double dm = norm(d);
        V3d rh = d / dm;
        double mr = dot(m, rh);
        double d3 = (dm * dm) * dm;
        V3d s = (3.0 * mr) * rh - m;
        return (coef * s) / d3;
    }
    // Analytic Jacobian: B_i = coef (3 (m.d) d_i / |d|^5 - m_i / |d|^3)
    // dB_i/dx_j = coef (3 (m_j d_i + (m.d) delta_ij + m_i d_j) / |d|^5
    //                   - 15 (m.d) d_i d_j / |d|^7)
    void jac(V3d r, double t, V3d& F, M3& J) const override {
        F = eval(r, t);
        V3d d = r - c;
        double d2 = abs2sum(d);
        double dm = std::sqrt(d2);
        double inv5 = 1.0 / ((d2 * d2) * dm);
        double inv7 = inv5 / d2;
        double md = dot(m, d);
        double dv[3] = {d.x, d.y, d.z}, mv[3] = {m.x, m.y, m.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double dij = (i == j) ? md : 0.0;
                J.a[3 * i + j] = coef * (3.0 * ((mv[j] * dv[i] + dij) + mv[i] * dv[j]) * inv5 -
                                         15.0 * md * dv[i] * dv[j] * inv7);
            }
    }
};

// Trilinear interpolation of a (3, nx, ny, nz) column-major array on a
// uniform grid, the reference's FieldInterpolator over linear_interp
// (src/utility/interpolation.jl:119-148,217-235).  Per axis:
//   u = (x - origin) * inv_dx, with inv_dx = 1/dx computed once;
//   FILL_NAN : u outside [0, n-1] -> NaN;  i = min(floor(u), n-2), f = u - i
//   CLAMP    : u clamped to [0, n-1];     i = min(floor(u), n-2), f = u - i
//   PERIODIC : i = floor(u), f = u - i, i = i mod n, i1 = (i+1) mod n
//              (period L = n*dx, PeriodicBC(endpoint=:exclusive))
// then lerp(a, b, f) = a + f*(b - a) along x, then y, then z.
template <class D>
struct GridField : Field {
    int64_t n[3];
    double x0[3], inv_dx[3];
    int bc;
    const D* data;  // (3, nx, ny, nz)

    struct Axis {
        int64_t i0, i1;
        double f;
        bool nan;
    };
    Axis axis(int a, double x) const {
        Axis r{0, 0, 0.0, false};
        double u = (x - x0[a]) * inv_dx[a];
        int64_t na = n[a];
        if (bc == TP_BC_PERIODIC) {
            double fl = std::floor(u);
            r.f = u - fl;
            int64_t i = (int64_t)fl % na;
            if (i < 0) i += na;
            r.i0 = i;
            r.i1 = (i + 1 == na) ? 0 : i + 1;
            return r;
        }
        double umax = (double)(na - 1);
        if (bc == TP_BC_CLAMP) {
            u = std::min(std::max(u, 0.0), umax);
        } else if (!(u >= 0.0 && u <= umax)) {
            r.nan = true;
            return r;
        }
        double fl = std::floor(u);
        int64_t i = (int64_t)fl;
        if (i > na - 2) i = na - 2;
        r.i0 = i;
        r.i1 = i + 1;
        r.f = u - (double)i;
        return r;
    }
    double at(int c, int64_t i, int64_t j, int64_t k) const {
        return (double)data[c + 3 * (i + n[0] * (j + n[1] * k))];
    }
    static double lerp(double a, double b, double f) { return a + f * (b - a); }

    V3d eval(V3d r, double) const override {
        Axis ax = axis(0, r.x), ay = axis(1, r.y), az = axis(2, r.z);
        if (ax.nan || ay.nan || az.nan) {
            double q = std::numeric_limits<double>::quiet_NaN();
            return {q, q, q};
        }
        double out[3];
        for (int c = 0; c < 3; ++c) {
            double c00 = lerp(at(c, ax.i0, ay.i0, az.i0), at(c, ax.i1, ay.i0, az.i0), ax.f);
            double c10 = lerp(at(c, ax.i0, ay.i1, az.i0), at(c, ax.i1, ay.i1, az.i0), ax.f);
            double c01 = lerp(at(c, ax.i0, ay.i0, az.i1), at(c, ax.i1, ay.i0, az.i1), ax.f);
            double c11 = lerp(at(c, ax.i0, ay.i1, az.i1), at(c, ax.i1, ay.i1, az.i1), ax.f);
            double c0 = lerp(c00, c10, ay.f);
            double c1 = lerp(c01, c11, ay.f);
            out[c] = lerp(c0, c1, az.f);
        }
        return {out[0], out[1], out[2]};
    }
    // Jacobian of the trilinear interpolant inside the cell (the derivative
    // ForwardDiff takes through linear_interp); clamped axes outside the
    // grid have zero derivative.
    void jac(V3d r, double t, V3d& F, M3& J) const override {
        F = eval(r, t);
        Axis ax = axis(0, r.x), ay = axis(1, r.y), az = axis(2, r.z);
        if (ax.nan || ay.nan || az.nan) {
            for (double& a : J.a) a = std::numeric_limits<double>::quiet_NaN();
            return;
        }
        double sx = inv_dx[0], sy = inv_dx[1], sz = inv_dx[2];
        if (bc == TP_BC_CLAMP) {
            double ux = (r.x - x0[0]) * inv_dx[0], uy = (r.y - x0[1]) * inv_dx[1],
                   uz = (r.z - x0[2]) * inv_dx[2];
            if (ux < 0.0 || ux > (double)(n[0] - 1)) sx = 0.0;
            if (uy < 0.0 || uy > (double)(n[1] - 1)) sy = 0.0;
            if (uz < 0.0 || uz > (double)(n[2] - 1)) sz = 0.0;
        }
        for (int c = 0; c < 3; ++c) {
            double v000 = at(c, ax.i0, ay.i0, az.i0), v100 = at(c, ax.i1, ay.i0, az.i0);
            double v010 = at(c, ax.i0, ay.i1, az.i0), v110 = at(c, ax.i1, ay.i1, az.i0);
            double v001 = at(c, ax.i0, ay.i0, az.i1), v101 = at(c, ax.i1, ay.i0, az.i1);
            double v011 = at(c, ax.i0, ay.i1, az.i1), v111 = at(c, ax.i1, ay.i1, az.i1);
            double fx = ax.f, fy = ay.f, fz = az.f;
            // d/dx
            double dx00 = v100 - v000, dx10 = v110 - v010, dx01 = v101 - v001, dx11 = v111 - v011;
            double dx0 = lerp(dx00, dx10, fy), dx1 = lerp(dx01, dx11, fy);
            J.a[3 * c + 0] = lerp(dx0, dx1, fz) * sx;
            // d/dy
            double c00 = lerp(v000, v100, fx), c10 = lerp(v010, v110, fx);
            double c01 = lerp(v001, v101, fx), c11 = lerp(v011, v111, fx);
            J.a[3 * c + 1] = lerp(c10 - c00, c11 - c01, fz) * sy;
            // d/dz
            double c0 = lerp(c00, c10, fy), c1 = lerp(c01, c11, fy);
            J.a[3 * c + 2] = (c1 - c0) * sz;
        }
    }
};

// Gridded fields beyond trilinear-uniform-Cartesian: build_interpolator with
// order 0 / 1 / 3, RectilinearGrid axes, StructuredGrid (spherical) and the
// 1-D / 2-D interpolants (src/utility/interpolation.jl:15-311) over
// FastInterpolations.jl v0.4 (constant_interp, linear_interp,
// cardinal_interp; a dependency absent here, restated from its documented
// behaviour and pinned on the reference's interpolation tests).
//   order 0   nearest node: floor(u + 1/2) on uniform axes, the closer node
//             on non-uniform ones (ties to the upper node)
//   order 1   cell i = min(floor(u), n - 2), f = u - i (non-uniform:
//             f = (x - c_i) / (c_{i+1} - c_i)); lerp a + f (b - a)
//   order 3   cardinal cubic (Catmull-Rom) Hermite on the same cell with
//             slopes (f_{i+1} - f_{i-1}) / 2; at the ends of a non-periodic
//             axis the three-point one-sided slope (-3 f0 + 4 f1 - f2) / 2,
//             mirrored at the top; two-node axes use the secant at both ends
//   periodic  exclusive: period n nodes; inclusive: period n - 1 nodes
//   spherical cart2sph (r = sqrt(x^2 + y^2 + z^2); theta = acos(z / r);
//             phi = atan(y, x) mapped to [0, 2pi)), r and theta fill NaN, phi
//             periodic inclusive; the (v_r, v_theta, v_phi) result goes
//             through sph2cartvec (src/utility/utility.jl:63-89); a scalar
//             grid (component 0) is returned as interpolated
// Templated on the scalar: double, or Dl3 (value and d/dx, d/dy, d/dz) for
// the Jacobian ForwardDiff would take.
struct Dl3 {
    double v, d[3];
};
inline double sval(double a) { return a; }
inline double sval(const Dl3& a) { return a.v; }
template <class S> inline S scst(double c);
template <> inline double scst<double>(double c) { return c; }
template <> inline Dl3 scst<Dl3>(double c) { return {c, {0.0, 0.0, 0.0}}; }
inline Dl3 operator+(const Dl3& a, const Dl3& b) { return {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
inline Dl3 operator-(const Dl3& a, const Dl3& b) { return {a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}}; }
inline Dl3 operator*(const Dl3& a, const Dl3& b) {
    Dl3 o{a.v * b.v, {0, 0, 0}};
    for (int k = 0; k < 3; ++k) o.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return o;
}
inline Dl3 operator/(const Dl3& a, const Dl3& b) {
    Dl3 o{a.v / b.v, {0, 0, 0}};
    for (int k = 0; k < 3; ++k) o.d[k] = (a.d[k] - o.v * b.d[k]) / b.v;
    return o;
}
inline Dl3 operator+(const Dl3& a, double c) { return {a.v + c, {a.d[0], a.d[1], a.d[2]}}; }
inline Dl3 operator+(double c, const Dl3& a) { return {c + a.v, {a.d[0], a.d[1], a.d[2]}}; }
inline Dl3 operator-(const Dl3& a, double c) { return {a.v - c, {a.d[0], a.d[1], a.d[2]}}; }
inline Dl3 operator-(double c, const Dl3& a) { return {c - a.v, {-a.d[0], -a.d[1], -a.d[2]}}; }
inline Dl3 operator*(const Dl3& a, double c) { return {a.v * c, {a.d[0] * c, a.d[1] * c, a.d[2] * c}}; }
inline Dl3 operator*(double c, const Dl3& a) { return {c * a.v, {c * a.d[0], c * a.d[1], c * a.d[2]}}; }
inline Dl3 operator/(const Dl3& a, double c) { return {a.v / c, {a.d[0] / c, a.d[1] / c, a.d[2] / c}}; }
inline double ssqrt(double a) { return std::sqrt(a); }
inline Dl3 ssqrt(const Dl3& a) {
    double r = std::sqrt(a.v), k = 0.5 / r;
    return {r, {a.d[0] * k, a.d[1] * k, a.d[2] * k}};
}
inline double sacos(double a) { return std::acos(a); }
inline Dl3 sacos(const Dl3& a) {
    double k = -1.0 / std::sqrt(1.0 - a.v * a.v);
    return {std::acos(a.v), {a.d[0] * k, a.d[1] * k, a.d[2] * k}};
}
inline double satan2(double y, double x) { return std::atan2(y, x); }
inline Dl3 satan2(const Dl3& y, const Dl3& x) {
    double den = x.v * x.v + y.v * y.v;
    Dl3 o{std::atan2(y.v, x.v), {0, 0, 0}};
    for (int k = 0; k < 3; ++k) o.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
    return o;
}
inline void ssincos(double a, double& s, double& c) {
    s = std::sin(a);
    c = std::cos(a);
}
inline void ssincos(const Dl3& a, Dl3& s, Dl3& c) {
    double sv = std::sin(a.v), cv = std::cos(a.v);
    s = {sv, {a.d[0] * cv, a.d[1] * cv, a.d[2] * cv}};
    c = {cv, {-(a.d[0] * sv), -(a.d[1] * sv), -(a.d[2] * sv)}};
}

template <class D>
struct GeneralGridField : Field {
    int64_t n[3];
    double x0[3], inv_dx[3];
    std::vector<double> coords[3];  // non-uniform axes (empty: uniform)
    int abc[3];                     // per-axis boundary
    int order, geom, ndim, dir;
    const D* data;                  // (3, n0, n1, n2)

    template <class S>
    struct Axis {
        int64_t i[4];
        S w[4];
        int k;
    };
    static int64_t wrap(int64_t i, int64_t m) {
        int64_t r = i % m;
        return r < 0 ? r + m : r;
    }

    template <class S>
    static void cubic(const S& t, int64_t i, int64_t na, bool periodic, int64_t m, Axis<S>& o) {
        S t2 = t * t;
        S t3 = t2 * t;
        S h00 = (2.0 * t3 - 3.0 * t2) + 1.0;
        S h10 = (t3 - 2.0 * t2) + t;
        S h01 = 3.0 * t2 - 2.0 * t3;
        S h11 = t3 - t2;
        if (periodic || (i > 0 && i < na - 2)) {
            o.k = 4;
            for (int q = 0; q < 4; ++q) o.i[q] = periodic ? wrap(i - 1 + q, m) : i - 1 + q;
            o.w[0] = -0.5 * h10;
            o.w[1] = h00 - 0.5 * h11;
            o.w[2] = h01 + 0.5 * h10;
            o.w[3] = 0.5 * h11;
        } else if (na == 2) {
            o.k = 2;
            o.i[0] = 0;
            o.i[1] = 1;
            o.w[0] = (h00 - h10) - h11;
            o.w[1] = (h01 + h10) + h11;
        } else if (i == 0) {
            o.k = 3;
            for (int q = 0; q < 3; ++q) o.i[q] = q;
            o.w[0] = (h00 - 1.5 * h10) - 0.5 * h11;
            o.w[1] = h01 + 2.0 * h10;
            o.w[2] = 0.5 * h11 - 0.5 * h10;
        } else {  // i == na - 2
            o.k = 3;
            for (int q = 0; q < 3; ++q) o.i[q] = na - 3 + q;
            o.w[0] = 0.5 * h11 - 0.5 * h10;
            o.w[1] = h00 - 2.0 * h11;
            o.w[2] = (h01 + 0.5 * h10) + 1.5 * h11;
        }
    }

    template <class S>
    bool axis(int a, S x, Axis<S>& o) const {
        const int64_t na = n[a];
        if (na == 1) {
            o.k = 1;
            o.i[0] = 0;
            return true;
        }
        const int bc = abc[a];
        if (!coords[a].empty()) {
            const std::vector<double>& c = coords[a];
            double xv = sval(x);
            if (bc == TP_BC_CLAMP) {
                if (xv < c.front()) x = scst<S>(c.front());
                else if (xv > c.back()) x = scst<S>(c.back());
                xv = sval(x);
            } else if (!(xv >= c.front() && xv <= c.back())) {
                return false;
            }
            // the last node with c_i <= x, at most n - 2
            int64_t il = std::upper_bound(c.begin(), c.end(), xv) - c.begin() - 1;
            il = std::max<int64_t>(0, std::min<int64_t>(il, na - 2));
            if (order == TP_ORDER_CONSTANT) {
                o.k = 1;
                o.i[0] = (xv - c[il] < c[il + 1] - xv) ? il : il + 1;
                return true;
            }
            o.k = 2;
            o.i[0] = il;
            o.i[1] = il + 1;
            o.w[0] = (x - c[il]) / (c[il + 1] - c[il]);
            return true;
        }
        S u = (x - x0[a]) * inv_dx[a];
        const bool periodic = bc == TP_BC_PERIODIC || bc == TP_BC_PERIODIC_INCLUSIVE;
        const int64_t m = bc == TP_BC_PERIODIC ? na : na - 1;
        const double umax = (double)(na - 1);
        if (order == TP_ORDER_CONSTANT) {
            double uv = sval(u);
            int64_t i;
            if (periodic) {
                i = wrap((int64_t)std::floor(uv + 0.5), m);
            } else {
                if (bc == TP_BC_CLAMP) uv = std::min(std::max(uv, 0.0), umax);
                else if (!(uv >= 0.0 && uv <= umax)) return false;
                i = (int64_t)std::floor(uv + 0.5);
            }
            o.k = 1;
            o.i[0] = i;
            return true;
        }
        int64_t i;
        S f;
        if (periodic) {
            double fl = std::floor(sval(u));
            f = u - fl;
            i = wrap((int64_t)fl, m);
        } else {
            double uv = sval(u);
            if (bc == TP_BC_CLAMP) {
                if (uv < 0.0) u = scst<S>(0.0);
                else if (uv > umax) u = scst<S>(umax);
            } else if (!(uv >= 0.0 && uv <= umax)) {
                return false;
            }
            i = std::min<int64_t>((int64_t)std::floor(sval(u)), na - 2);
            f = u - (double)i;
        }
        if (order == TP_ORDER_CUBIC) {
            cubic(f, i, na, periodic, m, o);
            return true;
        }
        o.k = 2;
        o.i[0] = i;
        o.i[1] = (bc == TP_BC_PERIODIC && i + 1 == na) ? 0 : i + 1;
        o.w[0] = f;
        return true;
    }

    template <class S, class V>
    S combine(const Axis<S>& a, const V* v) const {
        if (a.k == 1) return scst<S>(0.0) + v[0];
        if (order == TP_ORDER_LINEAR) return v[0] + a.w[0] * (v[1] - v[0]);
        S acc = a.w[0] * v[0] + a.w[1] * v[1];
        for (int q = 2; q < a.k; ++q) acc = acc + a.w[q] * v[q];
        return acc;
    }

    double node(int c, int64_t i, int64_t j, int64_t k) const {
        return (double)data[c + 3 * (i + n[0] * (j + n[1] * k))];
    }

    template <class S>
    bool interp(const S q[3], S out[3]) const {
        Axis<S> A[3];
        bool ok = axis(0, q[0], A[0]);
        ok = axis(1, q[1], A[1]) && ok;
        ok = axis(2, q[2], A[2]) && ok;
        if (!ok) return false;
        for (int c = 0; c < 3; ++c) {
            S cz[4] = {};
            for (int kz = 0; kz < A[2].k; ++kz) {
                S cy[4] = {};
                for (int ky = 0; ky < A[1].k; ++ky) {
                    double vx[4] = {0.0, 0.0, 0.0, 0.0};
                    for (int kx = 0; kx < A[0].k; ++kx) vx[kx] = node(c, A[0].i[kx], A[1].i[ky], A[2].i[kz]);
                    cy[ky] = combine<S, double>(A[0], vx);
                }
                cz[kz] = combine<S, S>(A[1], cy);
            }
            out[c] = combine<S, S>(A[2], cz);
        }
        return true;
    }

    template <class S>
    bool evaluate(const S r[3], S out[3]) const {
        if (geom == TP_GRID_SPHERICAL || geom == TP_GRID_SPHERICAL_SCALAR) {
            S rr = ssqrt((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]);
            S q[3];
            if (sval(rr) == 0.0) {
                q[0] = q[1] = q[2] = scst<S>(0.0);
            } else {
                q[0] = rr;
                q[1] = sacos(r[2] / rr);
                S ph = satan2(r[1], r[0]);
                if (sval(ph) < 0.0) ph = ph + 6.283185307179586;
                q[2] = ph;
            }
            S v[3];
            if (!interp(q, v)) return false;
            if (geom == TP_GRID_SPHERICAL_SCALAR) {  // a scalar: no basis conversion
                for (int c = 0; c < 3; ++c) out[c] = v[c];
                return true;
            }
            S st, ct, sp, cp;
            ssincos(q[1], st, ct);
            ssincos(q[2], sp, cp);
            out[0] = ((st * cp) * v[0] + (ct * cp) * v[1]) - sp * v[2];
            out[1] = ((st * sp) * v[0] + (ct * sp) * v[1]) + cp * v[2];
            out[2] = ct * v[0] - st * v[1];
            return true;
        }
        S q[3];
        if (ndim == 1) {
            q[0] = r[dir];
            q[1] = q[2] = scst<S>(0.0);
        } else {
            q[0] = r[0];
            q[1] = r[1];
            q[2] = r[2];
        }
        return interp(q, out);
    }

    V3d eval(V3d r, double) const override {
        double p[3] = {r.x, r.y, r.z}, o[3];
        if (!evaluate<double>(p, o)) {
            double nan = std::numeric_limits<double>::quiet_NaN();
            return {nan, nan, nan};
        }
        return {o[0], o[1], o[2]};
    }
    void jac(V3d r, double, V3d& F, M3& J) const override {
        Dl3 p[3] = {{r.x, {1, 0, 0}}, {r.y, {0, 1, 0}}, {r.z, {0, 0, 1}}}, o[3];
        if (!evaluate<Dl3>(p, o)) {
            double nan = std::numeric_limits<double>::quiet_NaN();
            F = {nan, nan, nan};
            for (double& a : J.a) a = nan;
            return;
        }
        F = {o[0].v, o[1].v, o[2].v};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) J.a[3 * i + j] = o[i].d[j];
    }
};

// LazyTimeInterpolator (src/utility/interpolation.jl:337-430): snapshots at
// sorted times; k = searchsortedlast(times, t); k == 0 or k == n clamp to the
// first / last snapshot, otherwise (1 - w) F_k + w F_{k+1}, w = (t - t_k) /
// (t_{k+1} - t_k); the Jacobian blends the snapshot Jacobians, derivative_t
// is (F_{k+1} - F_k) / (t_{k+1} - t_k) inside and zero outside.
struct SeriesField : Field {
    std::vector<double> times;
    std::vector<std::unique_ptr<Field>> snaps;
    int64_t index(double t) const { return std::upper_bound(times.begin(), times.end(), t) - times.begin(); }
    V3d eval(V3d r, double t) const override {
        int64_t k = index(t), n = (int64_t)times.size();
        if (k == 0) return snaps[0]->eval(r, t);
        if (k >= n) return snaps[n - 1]->eval(r, t);
        double w = (t - times[k - 1]) / (times[k] - times[k - 1]);
        V3d a = snaps[k - 1]->eval(r, t), b = snaps[k]->eval(r, t);
        return (1.0 - w) * a + w * b;
    }
    void jac(V3d r, double t, V3d& F, M3& J) const override {
        int64_t k = index(t), n = (int64_t)times.size();
        if (k == 0 || k >= n) {
            snaps[k == 0 ? 0 : n - 1]->jac(r, t, F, J);
            return;
        }
        double w = (t - times[k - 1]) / (times[k] - times[k - 1]);
        V3d Fa, Fb;
        M3 Ja, Jb;
        snaps[k - 1]->jac(r, t, Fa, Ja);
        snaps[k]->jac(r, t, Fb, Jb);
        F = (1.0 - w) * Fa + w * Fb;
        for (int q = 0; q < 9; ++q) J.a[q] = (1.0 - w) * Ja.a[q] + w * Jb.a[q];
    }
    V3d dtime(V3d r, double t) const override {
        int64_t k = index(t), n = (int64_t)times.size();
        if (k == 0 || k >= n) return {0.0, 0.0, 0.0};
        V3d a = snaps[k - 1]->eval(r, t), b = snaps[k]->eval(r, t);
        return (b - a) / (times[k] - times[k - 1]);
    }
};

// A field given by C callbacks (the tests' Julia closures restated in Python).
typedef void (*field_cb)(const double* x, double t, double* out, void* user);
typedef void (*jac_cb)(const double* x, double t, double* out9, void* user);
struct CallbackField : Field {
    field_cb f;
    jac_cb jf;
    void* user;
    V3d eval(V3d r, double t) const override {
        double x[3] = {r.x, r.y, r.z}, o[3];
        f(x, t, o, user);
        return {o[0], o[1], o[2]};
    }
    // dF/dt by a central difference (the tests' closures are smooth in t;
    // ForwardDiff.derivative takes it exactly)
    V3d dtime(V3d r, double t) const override {
        double h = 1.0e-6 * std::max(std::fabs(t), 1.0e-12);
        V3d a = eval(r, t + h), b = eval(r, t - h);
        return (a - b) / (2.0 * h);
    }
    void jac(V3d r, double t, V3d& F, M3& J) const override {
        F = eval(r, t);
        if (jf) {
            double x[3] = {r.x, r.y, r.z};
            jf(x, t, J.a, user);
        } else {
            for (double& a : J.a) a = 0.0;
        }
    }
};

// ---------------------------------------------------------------- termination
typedef int (*outside_cb)(const double* u, int len, double t, void* user);
struct Term {
    tp_term_desc d;
    outside_cb cb = nullptr;
    void* user = nullptr;
    bool any() const { return d.flags != 0 || cb != nullptr; }
    // isoutside(u, p, t) with u = (r, v) (full orbit) or (X, v_par) (GC)
    bool outside(const double* u, int len, double t) const {
        if (cb) return cb(u, len, t, user) != 0;
        int f = d.flags;
        if (f & TP_TERM_NAN)
            for (int k = 0; k < len; ++k)
                if (std::isnan(u[k])) return true;
        if (f & TP_TERM_SHELL) {
            double r = std::sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
            if (r < d.rmin || r > d.rmax) return true;
        }
        if (f & TP_TERM_BOX)
            for (int c = 0; c < 3; ++c)
                if (u[c] < d.lo[c] || u[c] > d.hi[c]) return true;
        if (f & TP_TERM_TIME)
            if (t > d.tmax) return true;
        return false;
    }
};

// ---------------------------------------------------------------- Boris core
// boris_velocity_update, src/boris/boris.jl:19-31
inline V3d boris_velocity_update(V3d v, V3d E, V3d B, double qdt_2m) {
    V3d t_rotate = qdt_2m * B;
    double t_mag2 = abs2sum(t_rotate);
    V3d s_rotate = (2.0 * t_rotate) / (1.0 + t_mag2);
    V3d vm = v + qdt_2m * E;
    V3d vp_ = vm + cross(vm, t_rotate);
    V3d vplus = vm + cross(vp_, s_rotate);
    return vplus + qdt_2m * E;
}

struct Params {
    double q2m, m;
    const Field* E;
    const Field* B;
};

// update_velocity, src/boris/boris.jl:38-45
struct BorisUpdater {
    V3d operator()(V3d v, V3d r, double dt, double t, const Params& p) const {
        V3d E = p.E->eval(r, t);
        V3d B = p.B->eval(r, t);
        double qdt_2m = p.q2m * 0.5 * dt;
        return boris_velocity_update(v, E, B, qdt_2m);
    }
};

// Portable sin / cos / atan2, built from +, -, *, / and sqrt only, so that the
// kernels and this restatement agree bit for bit.  Used for the hybrid's
// gyrophase (its step and mode decisions amplify last-bit differences) and
// in place of the reference's atan / sincos in the closed-form Multistep
// rotation (src/boris/multistep_boris.jl:110-119): Julia's, glibc's and
// CUDA's libm differ in the last bit, which a 1e4-step orbit amplifies.
//   sincos  Cody-Waite reduction by pi/2 (pi/2 split in three parts), then the
//           Taylor series of sin and cos on [-pi/4, pi/4] to degree 21 / 22
//   atan    for t in [0, 1]: up to two half-angle reductions tan(a/2) =
//           t / (1 + std::sqrt(1 + t^2)) to t <= tan(pi/16), then the Taylor
//           series to degree 29
inline void psincos(double x, double& s, double& c) {
    const double P1 = 1.570796325802803, P2 = 9.920935791635221e-10, P3 = 5.170182981794105e-19;
    const double kf = std::nearbyint(x * 0.6366197723675814);
    const double r = ((x - kf * P1) - kf * P2) - kf * P3;
    const double r2 = r * r;
    double ps = -1.0 / 51090942171709440000.0;
    ps = 1.0 / 121645100408832000.0 + r2 * ps;
    ps = -1.0 / 355687428096000.0 + r2 * ps;
    ps = 1.0 / 1307674368000.0 + r2 * ps;
    ps = -1.0 / 6227020800.0 + r2 * ps;
    ps = 1.0 / 39916800.0 + r2 * ps;
    ps = -1.0 / 362880.0 + r2 * ps;
    ps = 1.0 / 5040.0 + r2 * ps;
    ps = -1.0 / 120.0 + r2 * ps;
    ps = 1.0 / 6.0 + r2 * ps;
    const double sr = r - (r * r2) * ps;
    double pc = 1.0 / 1124000727777607680000.0;
    pc = -1.0 / 2432902008176640000.0 + r2 * pc;
    pc = 1.0 / 6402373705728000.0 + r2 * pc;
    pc = -1.0 / 20922789888000.0 + r2 * pc;
    pc = 1.0 / 87178291200.0 + r2 * pc;
    pc = -1.0 / 479001600.0 + r2 * pc;
    pc = 1.0 / 3628800.0 + r2 * pc;
    pc = -1.0 / 40320.0 + r2 * pc;
    pc = 1.0 / 720.0 + r2 * pc;
    pc = -1.0 / 24.0 + r2 * pc;
    pc = 0.5 + r2 * pc;
    const double cr = 1.0 - r2 * pc;
    const int q = (int)((long long)kf & 3);
    if (q == 0) {
        s = sr;
        c = cr;
    } else if (q == 1) {
        s = cr;
        c = -sr;
    } else if (q == 2) {
        s = -sr;
        c = -cr;
    } else {
        s = -cr;
        c = sr;
    }
}

inline double patan01(double t) {
    // halve the angle (tan(a/2) = t / (1 + sqrt(1 + t^2))) until |u| <= tan(pi/16)
    double u = t, scale = 1.0;
    if (u > 0.19891236737965800) {
        u = u / (1.0 + std::sqrt(1.0 + u * u));
        scale = 2.0;
    }
    if (u > 0.19891236737965800) {
        u = u / (1.0 + std::sqrt(1.0 + u * u));
        scale = 4.0;
    }
    const double u2 = u * u;
    double p = -1.0 / 29.0;
    p = 1.0 / 27.0 + u2 * p;
    p = -1.0 / 25.0 + u2 * p;
    p = 1.0 / 23.0 + u2 * p;
    p = -1.0 / 21.0 + u2 * p;
    p = 1.0 / 19.0 + u2 * p;
    p = -1.0 / 17.0 + u2 * p;
    p = 1.0 / 15.0 + u2 * p;
    p = -1.0 / 13.0 + u2 * p;
    p = 1.0 / 11.0 + u2 * p;
    p = -1.0 / 9.0 + u2 * p;
    p = 1.0 / 7.0 + u2 * p;
    p = -1.0 / 5.0 + u2 * p;
    p = 1.0 / 3.0 + u2 * p;
    const double a = u - (u * u2) * p;
    return scale * a;
}

inline double patan2(double y, double x) {
    if (x == 0.0 && y == 0.0) return 0.0;
    const double ax = std::fabs(x), ay = std::fabs(y);
    double a = (ay <= ax) ? patan01(ay / ax) : 1.5707963267948966 - patan01(ax / ay);
    if (x < 0.0) a = 3.141592653589793 - a;
    return (y < 0.0) ? -a : a;
}

// update_velocity_multistep, src/boris/multistep_boris.jl:65-142
// (@muladd fuses the scalar a*b+c forms: the Taylor coefficients and cos(2n alpha))
struct MultistepUpdater {
    int N;  // gyrophase correction order 2, 4, 6
    int n;  // subcycles
    V3d operator()(V3d v, V3d r, double dt, double t, const Params& p) const {
        V3d E = p.E->eval(r, t);
        V3d B = p.B->eval(r, t);
        double factor = p.q2m * dt / (double)(2 * n);
        V3d t_n = factor * B;
        V3d e_n = factor * E;
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
        double t_n_mag = std::sqrt(t_n_mag2);
        double c1, c2, c3, c6;
        double nd = (double)n;
        if (t_n_mag < 1.0e-4) {  // TN_MAG_THRESHOLD, src/boris/boris.jl:3
            c1 = std::fma(-(2.0 * nd * nd), t_n_mag2, 1.0);
            double n_term1 = 2.0 * nd;
            double n_term3 = 4.0 * nd * nd * nd;
            c2 = std::fma(-((n_term1 + n_term3) / 3.0), t_n_mag2, n_term1);
            c3 = std::fma(-((4.0 * nd * nd + 2.0 * nd * nd * nd * nd) / 3.0), t_n_mag2,
                          2.0 * nd * nd);
            c6 = (n_term1 + n_term3) / 3.0;
        } else {
            double alpha = patan2(t_n_mag, 1.0);  // atan(t_n_mag)
            double s, c;
            psincos(nd * alpha, s, c);  // sincos(n * alpha)
            double s2 = 2.0 * s * c;
            double cc = std::fma(c, c, -(s * s));
            c1 = cc;
            c2 = s2 / t_n_mag;
            c3 = 2.0 * s * s / t_n_mag2;
            c6 = (2.0 * nd - c2) / t_n_mag2;
        }
        double c4 = c2, c5 = c3;
        double v_dot_t = dot(v, t_n);
        double e_dot_t = dot(e_n, t_n);
        V3d v_cross_t = cross(v, t_n);
        V3d e_cross_t = cross(e_n, t_n);
        V3d out = c1 * v + c2 * v_cross_t;
        out = out + (c3 * v_dot_t) * t_n;
        out = out + c4 * e_n;
        out = out + c5 * e_cross_t;
        out = out + (c6 * e_dot_t) * t_n;
        return out;
    }
};

// Julia round(Int, x): round half to even
inline int64_t jl_round(double x) { return (int64_t)std::nearbyint(x); }

// _calculate_nout, src/boris/boris.jl:383-403
inline int64_t calculate_nout(int64_t nt, int64_t ssi, bool save_start, bool save_end,
                              bool save_everystep) {
    int64_t nout = 0;
    if (save_start) nout += 1;
    if (save_everystep) {
        int64_t steps = nt / ssi;
        bool last_is_step = (nt > 0) && (nt % ssi == 0);
        nout += steps;
        if (!save_end && last_is_step) nout -= 1;
        if (save_end && !last_is_step) nout += 1;
    } else if (save_end) {
        nout += 1;
    }
    return nout;
}

// One trajectory's output.
struct Traj {
    std::vector<double> t;
    std::vector<double> u;  // width per save
    int retcode = TP_RET_DEFAULT;
    int64_t nsteps = 0;
};

// get_magnetic_properties, src/utility/utility.jl:409-422, with _get_curvature
// (:379-384): grad|B| = JB' b, kappa = (JB b + b (-grad|B| . b)) / |B|
struct MagProps {
    V3d B, gradB, kappa, bh;
    double Bmag;
};
inline MagProps magnetic_properties(const Field& Bf, V3d r, double t) {
    MagProps m;
    M3 J;
    Bf.jac(r, t, m.B, J);
    m.Bmag = norm(m.B);
    if (m.Bmag == 0.0) {
        m.gradB = m.kappa = m.bh = V3d{0.0, 0.0, 0.0};
        return m;
    }
    V3d b = m.B / m.Bmag;
    m.bh = b;
    m.gradB = {(J(0, 0) * b.x + J(1, 0) * b.y) + J(2, 0) * b.z, (J(0, 1) * b.x + J(1, 1) * b.y) + J(2, 1) * b.z,
               (J(0, 2) * b.x + J(1, 2) * b.y) + J(2, 2) * b.z};
    V3d Jb{(J(0, 0) * b.x + J(0, 1) * b.y) + J(0, 2) * b.z, (J(1, 0) * b.x + J(1, 1) * b.y) + J(1, 2) * b.z,
           (J(2, 0) * b.x + J(2, 1) * b.y) + J(2, 2) * b.z};
    m.kappa = (Jb + b * (-dot(m.gradB, b))) / m.Bmag;
    return m;
}

// the four work rates (P_par, P_fermi, P_grad, P_betatron) of
// get_work_rates (src/equations.jl:394-441) and get_work_rates_gc (:445-480)
inline void work_terms(const MagProps& mp, V3d E, V3d dBdt, double q, double m, double vpar, double mu,
                       double* W) {
    W[0] = q * vpar * dot(E, mp.bh);
    W[1] = (m * (vpar * vpar) / mp.Bmag) * dot(cross(mp.bh, mp.kappa), E);
    W[2] = (mu / mp.Bmag) * dot(cross(mp.bh, mp.gradB), E);
    W[3] = mu * dot(dBdt, mp.bh);
}

inline void work_rates(const Params& p, V3d r, V3d v, double t, double* W) {
    double q = p.q2m * p.m;
    V3d E = p.E->eval(r, t);
    MagProps mp = magnetic_properties(*p.B, r, t);
    if (mp.Bmag == 0.0) {
        W[0] = W[1] = W[2] = W[3] = 0.0;
        return;
    }
    double vpar = dot(v, mp.bh);
    V3d vperp = v - vpar * mp.bh;
    double mu = p.m * dot(vperp, vperp) / (2.0 * mp.Bmag);
    work_terms(mp, E, p.B->dtime(r, t), q, p.m, vpar, mu, W);
}

// save flags: bit 0 = E and B (save_fields), bit 1 = work rates (save_work)
inline void push_save(Traj& out, const Params& p, int save_fields, V3d r, V3d v, double t) {
    out.t.push_back(t);
    double s[6] = {r.x, r.y, r.z, v.x, v.y, v.z};
    out.u.insert(out.u.end(), s, s + 6);
    if (save_fields & 1) {  // _prepare_saved_data, src/boris/boris.jl:405-427
        V3d E = p.E->eval(r, t), B = p.B->eval(r, t);
        double f[6] = {E.x, E.y, E.z, B.x, B.y, B.z};
        out.u.insert(out.u.end(), f, f + 6);
    }
    if (save_fields & 2) {  // boris.jl:429-437
        double w[4];
        work_rates(p, r, v, t, w);
        out.u.insert(out.u.end(), w, w + 4);
    }
}

struct FixedOpts {
    double t0, t1, dt;
    int64_t nt, nout, ssi;
    bool save_start, save_end, save_everystep;
    int save_fields;  // bit 0: E and B, bit 1: work rates
};

// _boris_single + _boris_loop!, src/boris/boris.jl:445-557
template <class Upd>
void boris_single(const Upd& upd, const Params& p, const FixedOpts& o, const Term& term,
                  const double* u0, Traj& out) {
    const double dt = o.dt;
    int64_t iout = 0;
    V3d r{u0[0], u0[1], u0[2]};
    V3d v{u0[3], u0[4], u0[5]};
    if (o.save_start) {
        iout += 1;
        push_save(out, p, o.save_fields, r, v, o.t0);
    }
    // push velocity back in time by 1/2 dt (boris.jl:514)
    v = upd(v, r, -0.5 * dt, o.t0, p);

    // _boris_loop! (boris.jl:445-478)
    int64_t it = 1;
    double t = o.t0 - 0.5 * dt;
    bool terminated = false;
    V3d v_prev = v;
    while (it <= o.nt) {
        v_prev = v;
        t += dt;
        v = upd(v, r, dt, t, p);
        V3d r_next = r + v * dt;
        double t_next = t + 0.5 * dt;
        if (term.any()) {
            double xv[6] = {r_next.x, r_next.y, r_next.z, v.x, v.y, v.z};
            if (term.outside(xv, 6, t_next)) {
                terminated = true;
                break;
            }
        }
        if (o.save_everystep && (it - 1) > 0 && (it - 1) % o.ssi == 0) {
            iout += 1;
            if (iout <= o.nout) {
                double t_current = t - 0.5 * dt;
                V3d v_save = upd(v_prev, r, 0.5 * dt, t_current, p);
                push_save(out, p, o.save_fields, r, v_save, t_current);
            }
        }
        r = r_next;
        it += 1;
    }
    int64_t final_step = it - 1;
    if (terminated) v = v_prev;  // return it - 1, iout, r, v_prev  (boris.jl:460)
    out.nsteps = final_step;

    bool should_save_final = false;
    if (o.save_end)
        should_save_final = true;
    else if (o.save_everystep && final_step > 0 && final_step % o.ssi == 0)
        should_save_final = true;

    if (iout < o.nout && should_save_final) {
        // @muladd: tspan[1] + final_step*dt and tspan[1] + (final_step - 0.5)*dt are fused
        double t_final = (final_step == o.nt) ? o.t1 : std::fma((double)final_step, dt, o.t0);
        if (iout == 0 || out.t.back() < t_final) {
            iout += 1;
            double dt_final = t_final - std::fma((double)final_step - 0.5, dt, o.t0);
            V3d v_final = upd(v, r, dt_final, t_final, p);
            push_save(out, p, o.save_fields, r, v_final, t_final);
        }
    }
    out.retcode = (iout < o.nout) ? TP_RET_TERMINATED : TP_RET_SUCCESS;
}

// _adaptive_boris_single, src/boris/adaptive_boris.jl:145-266
// step_cap (extension): stop after that many steps with retcode MaxIters.
template <class Upd>
void adaptive_single(const Upd& upd, const Params& p, double t0, double t1, double safety,
                     int64_t ssi, bool save_start, bool save_end, bool save_everystep,
                     int save_fields, int64_t step_cap, const Term& term, const double* u0,
                     Traj& out) {
    const double twopi = 6.283185307179586;  // Float64(2pi)
    double sgn = (t1 - t0) > 0 ? 1.0 : ((t1 - t0) < 0 ? -1.0 : 0.0);
    double C = (twopi * safety * sgn) / std::fabs(p.q2m);
    V3d r{u0[0], u0[1], u0[2]};
    V3d v{u0[3], u0[4], u0[5]};
    double t = t0;
    double ttotal = t1 - t0;
    if (save_start) push_save(out, p, save_fields, r, v, t);
    double Bmag = norm(p.B->eval(r, t));
    double dt = C / Bmag;
    v = upd(v, r, -0.5 * dt, t, p);
    int64_t it = 1;
    bool should_save_final = save_end;
    int ret = TP_RET_SUCCESS;
    int64_t steps = 0;
    while (std::fabs(t - t0) < std::fabs(ttotal)) {
        if (step_cap > 0 && steps >= step_cap) {
            ret = TP_RET_MAXITERS;
            break;
        }
        if (std::fabs(t + dt - t0) > std::fabs(ttotal)) {
            double dt_step = t1 - t;
            v = upd(v, r, 0.5 * dt, t, p);
            v = upd(v, r, -0.5 * dt_step, t, p);
            dt = dt_step;
        }
        if (save_everystep && (it - 1) > 0 && (it - 1) % ssi == 0) {
            V3d v_save = upd(v, r, 0.5 * dt, t, p);
            push_save(out, p, save_fields, r, v_save, t);
        }
        double t_mid = t + 0.5 * dt;
        V3d v_new = upd(v, r, dt, t_mid, p);
        V3d r_next = r + v_new * dt;
        double t_next = t + dt;
        if (term.any()) {
            double xv[6] = {r_next.x, r_next.y, r_next.z, v_new.x, v_new.y, v_new.z};
            if (term.outside(xv, 6, t_next)) {
                should_save_final = true;
                ret = TP_RET_TERMINATED;
                break;
            }
        }
        r = r_next;
        t = t_next;
        v = v_new;
        steps += 1;
        Bmag = norm(p.B->eval(r, t));
        double dt_new = C / Bmag;
        v = upd(v, r, 0.5 * dt, t, p);
        v = upd(v, r, -0.5 * dt_new, t, p);
        dt = dt_new;
        it += 1;
        if (save_everystep && (it - 1) % ssi == 0) should_save_final = true;
    }
    if (should_save_final && (out.t.empty() || out.t.back() != t)) {
        V3d v_final = upd(v, r, 0.5 * dt, t, p);
        push_save(out, p, save_fields, r, v_final, t);
    }
    out.retcode = ret;
    out.nsteps = steps;
}

// ---------------------------------------------------------------- guiding centre
struct GCParams {
    double q, q2m, mu;
    const Field* E;
    const Field* B;
};

struct GCState {
    double y[4];
};

// get_gc_derivatives, src/equations.jl:329-360 (with get_B_parameters, :239-247)
inline GCState gc_rhs(const GCState& s, const GCParams& p, double t) {
    V3d X{s.y[0], s.y[1], s.y[2]};
    V3d E = p.E->eval(X, t);
    V3d B;
    M3 J;
    p.B->jac(X, t, B, J);
    double Bmag = norm(B);
    V3d bh = B / Bmag;
    // grad|B| = JB' * bhat
    V3d gB{(J(0, 0) * bh.x + J(1, 0) * bh.y) + J(2, 0) * bh.z,
           (J(0, 1) * bh.x + J(1, 1) * bh.y) + J(2, 1) * bh.z,
           (J(0, 2) * bh.x + J(1, 2) * bh.y) + J(2, 2) * bh.z};
    V3d curlB{J(2, 1) - J(1, 2), J(0, 2) - J(2, 0), J(1, 0) - J(0, 1)};
    V3d curlb = (curlB + cross(bh, gB)) / Bmag;
    V3d Bs = B + (s.y[3] / p.q2m) * curlb;
    V3d Es = E - (p.mu / p.q) * gB;
    double inv_Bpar = 1.0 / dot(bh, Bs);
    V3d v = (s.y[3] * Bs + cross(Es, bh)) * inv_Bpar;
    double du = dot((p.q2m * inv_Bpar) * Bs, Es);
    return {{v.x, v.y, v.z, du}};
}

inline GCState gadd(const GCState& a, const GCState& b) {
    return {{a.y[0] + b.y[0], a.y[1] + b.y[1], a.y[2] + b.y[2], a.y[3] + b.y[3]}};
}
inline GCState gscale(double s, const GCState& a) {
    return {{s * a.y[0], s * a.y[1], s * a.y[2], s * a.y[3]}};
}

// update_rk4, src/gc/rk4_gc.jl:7-22
inline GCState update_rk4(const GCState& y, const GCParams& p, double dt, double t) {
    GCState k1 = gc_rhs(y, p, t);
    GCState yt = gadd(y, gscale(0.5 * dt, k1));
    GCState k2 = gc_rhs(yt, p, t + 0.5 * dt);
    yt = gadd(y, gscale(0.5 * dt, k2));
    GCState k3 = gc_rhs(yt, p, t + 0.5 * dt);
    yt = gadd(y, gscale(dt, k3));
    GCState k4 = gc_rhs(yt, p, t + dt);
    GCState sum = gadd(gadd(gadd(k1, gscale(2.0, k2)), gscale(2.0, k3)), k4);
    return gscale(dt / 6.0, sum);
}

// save flags: bit 0 = E and B, bit 1 = work rates (get_work_rates_gc)
inline void push_gc_save(Traj& out, const GCParams& p, int save_fields, const GCState& s,
                         double t) {
    out.t.push_back(t);
    out.u.insert(out.u.end(), s.y, s.y + 4);
    V3d X{s.y[0], s.y[1], s.y[2]};
    if (save_fields & 1) {  // _prepare_saved_data_gc, src/gc/gc_solver.jl:233-248
        V3d E = p.E->eval(X, t), B = p.B->eval(X, t);
        double f[6] = {E.x, E.y, E.z, B.x, B.y, B.z};
        out.u.insert(out.u.end(), f, f + 6);
    }
    if (save_fields & 2) {
        double w[4];
        V3d E = p.E->eval(X, t);
        MagProps mp = magnetic_properties(*p.B, X, t);
        if (mp.Bmag == 0.0) {
            w[0] = w[1] = w[2] = w[3] = 0.0;
        } else {
            work_terms(mp, E, p.B->dtime(X, t), p.q, p.q / p.q2m, s.y[3], p.mu, w);
        }
        out.u.insert(out.u.end(), w, w + 4);
    }
}

struct GCOpts {
    double t0, t1, dt;
    bool dt_given;
    int64_t nt, nout, ssi, maxiters;
    bool save_start, save_end, save_everystep;
    int save_fields;  // bit 0: E and B, bit 1: work rates
    double abstol, reltol;
};

// _rk4!, src/gc/rk4_gc.jl:27-130 (the @fastmath loop fuses t0 + (it-1)*dt)
inline void rk4_single(const GCParams& p, const GCOpts& o, const Term& term, const double* y0,
                       Traj& out) {
    GCState xv{{y0[0], y0[1], y0[2], y0[3]}};
    int64_t iout = 0;
    if (o.save_start) {
        iout += 1;
        push_gc_save(out, p, o.save_fields, xv, o.t0);
    }
    int64_t it = 1;
    const double dt = o.dt;
    while (it <= o.nt && it <= o.maxiters) {
        double t = std::fma((double)(it - 1), dt, o.t0);
        GCState dx = update_rk4(xv, p, dt, t);
        GCState xn = gadd(xv, dx);
        if (term.any() && term.outside(xn.y, 4, t + dt)) break;
        xv = xn;
        if (o.save_everystep && (it % o.ssi == 0)) {
            iout += 1;
            if (iout <= o.nout) push_gc_save(out, p, o.save_fields, xv, t + dt);
        }
        it += 1;
    }
    int64_t final_step = it - 1;
    bool should_save_final = false;
    if (o.save_end)
        should_save_final = true;
    else if (o.save_everystep && final_step > 0 && final_step % o.ssi == 0)
        should_save_final = true;
    if (iout < o.nout && should_save_final) {
        double t_final = (final_step == o.nt) ? o.t1 : std::fma((double)final_step, dt, o.t0);
        if (iout == 0 || out.t.back() < t_final) {
            iout += 1;
            push_gc_save(out, p, o.save_fields, xv, t_final);
        }
    }
    if (it <= o.nt && it <= o.maxiters)
        out.retcode = TP_RET_TERMINATED;
    else if (it > o.maxiters)
        out.retcode = TP_RET_MAXITERS;
    else
        out.retcode = TP_RET_SUCCESS;
    out.nsteps = final_step;
}

// Dormand-Prince 5(4) tableau, src/gc/rk45_gc.jl:9-20
struct DP5 {
    static constexpr double c2 = 1.0 / 5, c3 = 3.0 / 10, c4 = 4.0 / 5, c5 = 8.0 / 9, c6 = 1.0;
    static constexpr double a21 = 1.0 / 5;
    static constexpr double a31 = 3.0 / 40, a32 = 9.0 / 40;
    static constexpr double a41 = 44.0 / 45, a42 = -56.0 / 15, a43 = 32.0 / 9;
    static constexpr double a51 = 19372.0 / 6561, a52 = -25360.0 / 2187, a53 = 64448.0 / 6561,
                            a54 = -212.0 / 729;
    static constexpr double a61 = 9017.0 / 3168, a62 = -355.0 / 33, a63 = 46732.0 / 5247,
                            a64 = 49.0 / 176, a65 = -5103.0 / 18656;
    static constexpr double a71 = 35.0 / 384, a72 = 0.0, a73 = 500.0 / 1113, a74 = 125.0 / 192,
                            a75 = -2187.0 / 6784, a76 = 11.0 / 84;
    static constexpr double b1 = 35.0 / 384, b3 = 500.0 / 1113, b4 = 125.0 / 192,
                            b5 = -2187.0 / 6784, b6 = 11.0 / 84;
    static constexpr double e1 = 71.0 / 57600, e3 = -71.0 / 16695, e4 = 71.0 / 1920,
                            e5 = -17253.0 / 339200, e6 = 22.0 / 525, e7 = -1.0 / 40;
};

// update_dp5, src/gc/rk45_gc.jl:7-47.  Linear combinations are summed left to
// right, each term a scalar times a vector, then scaled by dt; the stage times
// t + c_k*dt are fused by @muladd.
inline void update_dp5(const GCState& y, const GCParams& p, double dt, double t, GCState& dy,
                       GCState& err) {
    typedef DP5 D;
    GCState k1 = gc_rhs(y, p, t);
    GCState yt = gadd(y, gscale(dt, gscale(D::a21, k1)));
    GCState k2 = gc_rhs(yt, p, std::fma(D::c2, dt, t));
    yt = gadd(y, gscale(dt, gadd(gscale(D::a31, k1), gscale(D::a32, k2))));
    GCState k3 = gc_rhs(yt, p, std::fma(D::c3, dt, t));
    yt = gadd(y, gscale(dt, gadd(gadd(gscale(D::a41, k1), gscale(D::a42, k2)), gscale(D::a43, k3))));
    GCState k4 = gc_rhs(yt, p, std::fma(D::c4, dt, t));
    yt = gadd(y, gscale(dt, gadd(gadd(gadd(gscale(D::a51, k1), gscale(D::a52, k2)),
                                      gscale(D::a53, k3)),
                                 gscale(D::a54, k4))));
    GCState k5 = gc_rhs(yt, p, std::fma(D::c5, dt, t));
    yt = gadd(y, gscale(dt, gadd(gadd(gadd(gadd(gscale(D::a61, k1), gscale(D::a62, k2)),
                                           gscale(D::a63, k3)),
                                      gscale(D::a64, k4)),
                                 gscale(D::a65, k5))));
    GCState k6 = gc_rhs(yt, p, std::fma(D::c6, dt, t));
    yt = gadd(y, gscale(dt, gadd(gadd(gadd(gadd(gadd(gscale(D::a71, k1), gscale(D::a72, k2)),
                                                gscale(D::a73, k3)),
                                           gscale(D::a74, k4)),
                                      gscale(D::a75, k5)),
                                 gscale(D::a76, k6))));
    GCState k7 = gc_rhs(yt, p, t + dt);
    dy = gscale(dt, gadd(gadd(gadd(gadd(gscale(D::b1, k1), gscale(D::b3, k3)), gscale(D::b4, k4)),
                              gscale(D::b5, k5)),
                         gscale(D::b6, k6)));
    err = gscale(dt, gadd(gadd(gadd(gadd(gadd(gscale(D::e1, k1), gscale(D::e3, k3)),
                                         gscale(D::e4, k4)),
                                    gscale(D::e5, k5)),
                               gscale(D::e6, k6)),
                          gscale(D::e7, k7)));
}

// x^0.2 rounded to nearest, the step-size factor of rk45_gc.jl:151
// (`(1.0 / error_ratio)^0.2`, a Float64 `^`).  Julia's `^` and the C library's
// pow are accurate to about half an ulp but, within a small fraction of an
// ulp of a rounding tie, round either way; a one-ulp difference in the factor
// shifts every later step.  Both the oracle and the CUDA kernels therefore use
// this function: one Newton step for the real fifth root z = x^(1/5) from the
// library pow z0, with the residual z0^5 - x evaluated in double-double
// arithmetic (Dekker's exact product by fma; z0^5 - x is exact by Sterbenz's
// lemma), then the exponent correction x^(0.2 - 1/5) = 1 + d ln x for the
// float64 constant 0.2 = 1/5 + d, d = 2^-54 / 5.  The result is the correctly
// rounded x^0.2 unless x^0.2 lies within ~1e-30 relative of a tie.  Outside
// [1e-30, 1e30] (where the controller clamps the factor anyway) it returns z0.
inline double pow02_rn(double x) {
    double z0 = std::pow(x, 0.2);
    if (!(x >= 1.0e-30 && x <= 1.0e30) || !(z0 > 0.0) || std::isinf(z0)) return z0;
    double a = z0 * z0;
    double ae = std::fma(z0, z0, -a);
    double b = a * a;
    double be = std::fma(a, a, -b) + (2.0 * a) * ae;
    double c = b * z0;
    double ce = std::fma(b, z0, -c) + be * z0;
    double r = (c - x) + ce;
    double corr = -r / (5.0 * b);
    double t = (0.2 * 0x1p-54) * std::log(x);
    return z0 + (corr + z0 * t);
}

// _rk45!, src/gc/rk45_gc.jl:52-173 (inside @fastmath: the error scale and the
// sum of squares are fused multiply-adds)
inline void rk45_single(const GCParams& p, const GCOpts& o, const Term& term, const double* y0,
                        Traj& out) {
    const double safety = 0.9, max_growth = 5.0, min_growth = 0.2;
    GCState xv{{y0[0], y0[1], y0[2], y0[3]}};
    double t = o.t0;
    double dt;
    if (!o.dt_given) {
        V3d R{xv.y[0], xv.y[1], xv.y[2]};
        double Bmag = norm(p.B->eval(R, t));
        if (Bmag == 0.0 || p.q2m == 0.0) {
            dt = 1.0e-6;
        } else {
            double omega = std::fabs(p.q2m * Bmag);
            dt = 0.5 * 6.283185307179586 / omega;
        }
    } else {
        dt = o.dt;
    }
    if (o.save_start) push_gc_save(out, p, o.save_fields, xv, t);
    int64_t steps = 0;
    int ret = TP_RET_SUCCESS;
    while (t < o.t1 && steps < o.maxiters) {
        if (t + dt > o.t1) dt = o.t1 - t;
        GCState dx, E;
        update_dp5(xv, p, dt, t, dx, E);
        GCState yn = gadd(xv, dx);
        double sum_sq = 0.0;
        for (int k = 0; k < 4; ++k) {
            double sc = std::fma(std::max(std::fabs(xv.y[k]), std::fabs(yn.y[k])), o.reltol, o.abstol);
            double q = E.y[k] / sc;
            sum_sq = std::fma(q, q, sum_sq);
        }
        double error_ratio = 0.5 * std::sqrt(sum_sq);
        // `error_ratio <= 1.0` inside @fastmath: the no-NaN comparison accepts a
        // NaN ratio, after which isoutside sees the NaN state and terminates
        // (the reference's test_boundary.jl:84-95 expects Terminated there).
        if (!(error_ratio > 1.0)) {
            if (term.any() && term.outside(yn.y, 4, t + dt)) {
                ret = TP_RET_TERMINATED;
                break;
            }
            t += dt;
            xv = yn;
            if (o.save_everystep) push_gc_save(out, p, o.save_fields, xv, t);
            steps += 1;
        }
        double scale = (error_ratio == 0.0) ? max_growth : safety * pow02_rn(1.0 / error_ratio);
        scale = std::max(min_growth, std::min(scale, max_growth));
        dt *= scale;
        if (dt < 1.0e-14) break;
    }
    if (o.save_end && (out.t.empty() || out.t.back() != t)) push_gc_save(out, p, o.save_fields, xv, t);
    out.retcode = ret;
    out.nsteps = steps;
}

// get_perp_vector, src/utility/utility.jl:119-126
inline void get_perp_vector(V3d b, V3d& e1, V3d& e2) {
    V3d bh = b / norm(b);
    V3d v = std::fabs(bh.z) < 0.9 ? V3d{0.0, 0.0, 1.0} : V3d{0.0, 1.0, 0.0};
    V3d c = cross(v, bh);
    e1 = c / norm(c);
    e2 = cross(bh, e1);
}

// _get_gc_parameters, src/gc/gc.jl:13-39 -> (X, vpar, mu)
inline void gc_parameters(const double* xv, const Field& E, const Field& B, double q, double m,
                          double t, double* X_out, double* vpar_out, double* mu_out) {
    V3d x{xv[0], xv[1], xv[2]}, v{xv[3], xv[4], xv[5]};
    V3d bp = B.eval(x, t);
    double Bmp = norm(bp);
    V3d bhp = bp / Bmp;
    V3d rho = cross(bhp, v) / (q / m * Bmp);
    V3d X = x - rho;
    V3d b = B.eval(X, t);
    double Bmag = norm(b);
    V3d bh = b / Bmag;
    double vpar = dot(bh, v);
    V3d vperp = v - vpar * bh;
    V3d e = E.eval(X, t);
    V3d vE = cross(e, bh) / Bmag;
    V3d w = vperp - vE;
    double mu = m * dot(w, w) / (2.0 * Bmag);
    X_out[0] = X.x;
    X_out[1] = X.y;
    X_out[2] = X.z;
    *vpar_out = vpar;
    *mu_out = mu;
}


// ---------------------------------------------------------------- hybrid
// _hybrid_adaptive!, src/hybrid.jl:234-474, one trajectory.  Helpers:
// _get_gc_parameters with the gyrophase (src/gc/gc.jl:13-39), _gc_to_full
// (:128-154), adiabaticity_components (src/utility/utility.jl:554-577),
// _fo_dt (hybrid.jl:226-232), mod2pi with 2 pi carried as two doubles.
struct HybridOpts {
    double t0, t1, th_gc_fo, th_fo_gc, dtmin, dtmax, safety_fo, abstol, reltol;
    int64_t maxiters, check, ssi;
    int adia_mode;
    bool save_start, save_end, save_everystep;
};

struct HybridTraj {
    Traj traj;
    std::vector<double> at, av;  // adiabaticity checks: time; (value, mode) pairs
};


inline double mod2pi_d(double x) {
    const double hi = 6.283185307179586, lo = 2.4492935982947064e-16;
    double k = std::floor(x / hi);
    double r = std::fma(-k, hi, x);
    r = std::fma(-k, lo, r);
    if (r < 0.0) r = (r + hi) + lo;
    else if (r >= hi) r = (r - hi) - lo;
    return r;
}

inline void gc_params_phase(V3d x, V3d v, const Field& E, const Field& B, double q, double m, double t, V3d& X,
                            double& vpar, double& mu, double& phase) {
    V3d bp = B.eval(x, t);
    double Bmp = norm(bp);
    V3d bhp = bp / Bmp;
    V3d rho = cross(bhp, v) / (q / m * Bmp);
    X = x - rho;
    V3d b = B.eval(X, t);
    double Bmag = norm(b);
    V3d bh = b / Bmag;
    vpar = dot(bh, v);
    V3d vperp = v - vpar * bh;
    V3d e = E.eval(X, t);
    V3d vE = cross(e, bh) / Bmag;
    V3d w = vperp - vE;
    mu = m * dot(w, w) / (2.0 * Bmag);
    V3d e1, e2;
    get_perp_vector(bh, e1, e2);
    phase = patan2(dot(w, e2), dot(w, e1));
}

inline void gc_to_full(const GCState& s, const Field& Ef, const Field& Bf, double q, double m, double mu,
                       double t, double phase, V3d& x, V3d& v) {
    V3d R{s.y[0], s.y[1], s.y[2]};
    V3d E = Ef.eval(R, t), B = Bf.eval(R, t);
    double Bmag = norm(B);
    V3d bh = B / Bmag;
    V3d vE = cross(E, bh) / Bmag;
    double w = std::sqrt(2.0 * mu * Bmag / m);
    V3d e1, e2;
    get_perp_vector(bh, e1, e2);
    double sp, cp;
    psincos(phase, sp, cp);
    V3d vperp = w * (cp * e1 + sp * e2) + vE;
    v = s.y[3] * bh + vperp;
    double Om = q * Bmag / m;
    x = R + cross(bh, vperp) / Om;
}

inline void adiabaticity_components(const Field& Bf, V3d x, double q, double m, double mu, double t, double c[3]) {
    V3d B;
    M3 J;
    Bf.jac(x, t, B, J);
    double Bmag = norm(B);
    const double inf = std::numeric_limits<double>::infinity();
    if (Bmag == 0.0) {
        c[0] = c[1] = c[2] = inf;
        return;
    }
    double rho = std::sqrt(2.0 * mu * m / Bmag) / std::fabs(q);
    V3d bh = B / Bmag;
    V3d gB{(J(0, 0) * bh.x + J(1, 0) * bh.y) + J(2, 0) * bh.z, (J(0, 1) * bh.x + J(1, 1) * bh.y) + J(2, 1) * bh.z,
           (J(0, 2) * bh.x + J(1, 2) * bh.y) + J(2, 2) * bh.z};
    double gBm = norm(gB);
    double LB = gBm == 0.0 ? inf : Bmag / gBm;
    c[1] = rho / LB;
    V3d Jb{(J(0, 0) * bh.x + J(0, 1) * bh.y) + J(0, 2) * bh.z, (J(1, 0) * bh.x + J(1, 1) * bh.y) + J(1, 2) * bh.z,
           (J(2, 0) * bh.x + J(2, 1) * bh.y) + J(2, 2) * bh.z};
    V3d kap = (Jb + bh * (-dot(gB, bh))) / Bmag;
    c[0] = rho * norm(kap);
    double fro = 0.0;  // sum(abs2, JB), column-major
    bool first = true;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double a = J(i, j) * J(i, j);
            fro = first ? a : fro + a;
            first = false;
        }
    c[2] = rho * std::sqrt(fro) / Bmag;
}

inline double adia_select(const double c[3], int mode) {
    if (mode == TP_ADIA_CURVATURE) return c[0];
    if (mode == TP_ADIA_GRADB) return c[1];
    if (mode == TP_ADIA_JACOBIAN) return c[2];
    if (std::isnan(c[0]) || std::isnan(c[1])) return c[0] + c[1];
    return c[0] < c[1] ? c[1] : c[0];
}

inline void hybrid_single(const Params& p, const HybridOpts& o, const Term& term, const double* u0, bool save_adia,
                          HybridTraj& out) {
    const double two_pi = 6.283185307179586;
    const Field& Ef = *p.E;
    const Field& Bf = *p.B;
    const double q = p.q2m * p.m;
    const bool is_td = Ef.dtime({0, 0, 0}, 0.0).x != 0.0 || Ef.dtime({0, 0, 0}, 0.0).y != 0.0 ||
                       Ef.dtime({0, 0, 0}, 0.0).z != 0.0 || Bf.dtime({0, 0, 0}, 0.0).x != 0.0 ||
                       Bf.dtime({0, 0, 0}, 0.0).y != 0.0 || Bf.dtime({0, 0, 0}, 0.0).z != 0.0;
    BorisUpdater upd;
    auto fo_dt = [&](V3d r, double t) {
        double Bmag = norm(Bf.eval(r, t));
        double om = std::fabs(p.q2m) * Bmag;
        double dt = two_pi * o.safety_fo / om;
        return dt > o.dtmax ? o.dtmax : (dt < o.dtmin ? o.dtmin : dt);
    };
    auto push = [&](V3d x, V3d v, double t) {
        out.traj.t.push_back(t);
        double s[6] = {x.x, x.y, x.z, v.x, v.y, v.z};
        out.traj.u.insert(out.traj.u.end(), s, s + 6);
    };
    auto push_adia = [&](double t, double eps, bool gc) {
        if (!save_adia) return;
        out.at.push_back(t);
        out.av.push_back(eps);
        out.av.push_back(gc ? 0.0 : 1.0);
    };
    V3d r{u0[0], u0[1], u0[2]}, v{u0[3], u0[4], u0[5]};
    double t = o.t0;
    GCParams pg{q, p.q2m, 0.0, p.E, p.B};
    V3d X;
    double vpar, mu, phase;
    gc_params_phase(r, v, Ef, Bf, q, p.m, t, X, vpar, mu, phase);
    double c[3];
    adiabaticity_components(Bf, r, q, p.m, mu, t, c);
    double eps = adia_select(c, o.adia_mode);
    bool gc = eps < o.th_gc_fo;
    GCState xg{{0, 0, 0, 0}};
    double dt;
    if (gc) {
        xg = {{X.x, X.y, X.z, vpar}};
        pg.mu = mu;
        double Bmag = norm(Bf.eval(X, t));
        dt = 0.5 * two_pi / std::fabs(p.q2m * Bmag);
    } else {
        dt = fo_dt(r, t);
        v = upd(v, r, -0.5 * dt, t, p);
    }
    push_adia(t, eps, gc);
    if (o.save_start) push({u0[0], u0[1], u0[2]}, {u0[3], u0[4], u0[5]}, t);
    int64_t steps = 0, it = 1;
    int ret = TP_RET_SUCCESS;
    while (t < o.t1 && steps < o.maxiters) {
        if (gc) {
            if (it % o.check == 0) {
                adiabaticity_components(Bf, {xg.y[0], xg.y[1], xg.y[2]}, q, p.m, mu, t, c);
                eps = adia_select(c, o.adia_mode);
                push_adia(t, eps, true);
                if (eps >= o.th_gc_fo) {
                    gc = false;
                    gc_to_full(xg, Ef, Bf, q, p.m, mu, t, phase, r, v);
                    dt = fo_dt(r, t);
                    v = upd(v, r, -0.5 * dt, t, p);
                    continue;
                }
            }
            if (t + dt > o.t1) dt = o.t1 - t;
            GCState dx, Er;
            update_dp5(xg, pg, dt, t, dx, Er);
            GCState yn = gadd(xg, dx);
            double sum_sq = 0.0;
            for (int k = 0; k < 4; ++k) {
                double ax = std::fabs(xg.y[k]), ay = std::fabs(yn.y[k]);
                double sc = o.abstol + ((ax < ay) ? ay : ax) * o.reltol;
                double qk = Er.y[k] / sc;
                sum_sq = sum_sq + qk * qk;
            }
            double er = 0.5 * std::sqrt(sum_sq);
            if (std::isnan(er)) {
                ret = TP_RET_TERMINATED;
                break;
            }
            if (er <= 1.0) {
                if (term.any() && term.outside(yn.y, 4, t + dt)) break;
                t += dt;
                xg = yn;
                double Bs = norm(Bf.eval({xg.y[0], xg.y[1], xg.y[2]}, t));
                phase = mod2pi_d(phase - dt * (p.q2m * Bs));
                if (o.save_everystep && it % o.ssi == 0) {
                    V3d xs, vs;
                    gc_to_full(xg, Ef, Bf, q, p.m, mu, t, phase, xs, vs);
                    push(xs, vs, t);
                }
                steps += 1;
                it += 1;
            }
            double scale = (er == 0.0) ? 5.0 : 0.9 * pow02_rn(1.0 / er);
            scale = (scale < 5.0) ? scale : 5.0;
            scale = (0.2 < scale) ? scale : 0.2;
            dt *= scale;
            if (dt < 1.0e-14) break;
        } else {
            if (it % o.check == 0) {
                const double t_sync = is_td ? t : 0.0;
                V3d vs = upd(v, r, 0.5 * dt, t_sync, p);
                V3d Xf;
                double vparf, muf, phasef;
                gc_params_phase(r, vs, Ef, Bf, q, p.m, t, Xf, vparf, muf, phasef);
                adiabaticity_components(Bf, Xf, q, p.m, muf, t, c);
                eps = adia_select(c, o.adia_mode);
                push_adia(t, eps, false);
                if (eps < o.th_fo_gc) {
                    gc = true;
                    xg = {{Xf.x, Xf.y, Xf.z, vparf}};
                    pg.mu = muf;
                    mu = muf;
                    phase = phasef;
                    double Bmag = norm(Bf.eval(r, t));
                    dt = 0.5 * two_pi / std::fabs(p.q2m * Bmag);
                    continue;
                }
            }
            if (t + dt > o.t1) dt = o.t1 - t;
            V3d vprev = v;
            v = upd(v, r, dt, t + 0.5 * dt, p);
            V3d rn = r + v * dt;
            double tn = t + dt;
            double xvn[6] = {rn.x, rn.y, rn.z, v.x, v.y, v.z};
            if (term.any() && term.outside(xvn, 6, tn)) break;
            if (o.save_everystep && it - 1 > 0 && (it - 1) % o.ssi == 0) push(r, upd(vprev, r, 0.5 * dt, t, p), t);
            r = rn;
            t = tn;
            it += 1;
            steps += 1;
        }
    }
    if (o.save_end && (out.traj.t.empty() || out.traj.t.back() != t)) {
        if (gc) {
            V3d xs, vs;
            gc_to_full(xg, Ef, Bf, q, p.m, mu, t, phase, xs, vs);
            push(xs, vs, t);
        } else {
            const double t_final = is_td ? t : 0.0;
            push(r, upd(v, r, 0.5 * dt, t_final, p), t);
        }
    }
    out.traj.retcode = ret != TP_RET_SUCCESS ? ret : (steps >= o.maxiters ? TP_RET_MAXITERS : TP_RET_SUCCESS);
    out.traj.nsteps = steps;
}


// ---------------------------------------------------------------- detectors
// Virtual detectors of the Meshes extension (ext/TestParticleMeshesExt.jl:
// 98-491) over packed trajectories.  _signed_distance: (p - p0) . n for a
// plane or disk, |p - c| - r for a sphere; _is_valid_intersection: a disk
// crossing lies within the radius.  A segment crosses when s1 s2 < 0 or
// (s1 != 0 and s2 == 0), at f = s1 / (s1 - s2), t = muladd(f, t2 - t1, t1);
// the state there is the solution's linear interpolation (searchsortedlast,
// u_i + theta (u_{i+1} - u_i), as the reference tests' MockSol).
inline double det_sdist(const tp_surface& S, V3d p) {
    V3d v = p - V3d{S.point[0], S.point[1], S.point[2]};
    if (S.kind == TP_SURF_SPHERE) return norm(v) - S.radius;
    return dot(v, V3d{S.normal[0], S.normal[1], S.normal[2]});
}

inline bool det_valid(const tp_surface& S, V3d p) {
    if (S.kind != TP_SURF_DISK) return true;
    V3d d = p - V3d{S.point[0], S.point[1], S.point[2]};
    return dot(d, d) <= S.radius * S.radius;
}

inline void det_interp(const double* t, const double* u, int W, int64_t m, double tc, double s[6]) {
    int64_t i = std::upper_bound(t, t + m, tc) - t - 1;
    if (i < 0 || i >= m - 1) {
        const double* r = u + (i < 0 ? 0 : m - 1) * W;
        for (int c = 0; c < 6; ++c) s[c] = r[c];
        return;
    }
    double th = (tc - t[i]) / (t[i + 1] - t[i]);
    for (int c = 0; c < 6; ++c) s[c] = u[i * W + c] + th * (u[(i + 1) * W + c] - u[i * W + c]);
}

// Calls visit(state) for each valid crossing of trajectory (t, u, m) in time
// order; returns early when visit returns false.  first_zero: the first
// save lies on the surface (get_first_crossing returns it).
template <class Visit>
inline void det_walk(const double* t, const double* u, int W, int64_t m, const tp_surface& S, Visit visit,
                     bool* first_zero = nullptr) {
    if (m < 1) return;
    V3d p1{u[0], u[1], u[2]};
    double s1 = det_sdist(S, p1);
    if (first_zero) *first_zero = (s1 == 0.0);
    for (int64_t k = 0; k + 1 < m; ++k) {
        V3d p2{u[(k + 1) * W], u[(k + 1) * W + 1], u[(k + 1) * W + 2]};
        double s2 = det_sdist(S, p2);
        if (s1 * s2 < 0.0 || (s1 != 0.0 && s2 == 0.0)) {
            double f = s1 / (s1 - s2);
            V3d pc = p1 + f * (p2 - p1);
            if (det_valid(S, pc)) {
                double tc = std::fma(f, t[k + 1] - t[k], t[k]);
                double st[6];
                det_interp(t, u, W, m, tc, st);
                if (!visit(st)) return;
            }
        }
        s1 = s2;
        p1 = p2;
    }
}

}  // namespace orc
