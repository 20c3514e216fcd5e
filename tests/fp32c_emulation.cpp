// CPU emulation of the FP32C MultistepBoris4(n=2) push in the Earth dipole,
// with the arithmetic of each ingredient switchable between float32 and
// float64.  Test infrastructure for tests/test_fp32c_design.py: it shows,
// on the CPU and against the float64 oracle, which float32 roundings make
// the final-position error of the dipole ensemble, and so why the device's
// FP32C analytic-field kernels (fp32c_common.cuh) keep the field and the
// velocity in float64 while the rotation factors stay float32.  It follows
// the device arithmetic operation by operation but is not bit-exact with it
// (the compiler's contractions differ); the test compares error statistics.
//
//   g++ -O2 -fopenmp -ffp-contract=off -shared -fPIC -o fp32c_emulation.so fp32c_emulation.cpp
#include <cmath>
#include <cstdint>

namespace {

struct F3 {
    float x, y, z;
};
struct D3 {
    double x, y, z;
};
inline float dotf(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 crossf(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 crossd(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// (hi, lo) += d: TwoSum then Fast2Sum
inline void cadd(float& hi, float& lo, float d) {
    float s = hi + d;
    float bb = s - hi;
    float e = (hi - (s - bb)) + (d - bb);
    e = e + lo;
    float h = s + e;
    lo = e - (h - s);
    hi = h;
}

struct State {
    float hi[3], lo[3];  // compensated position
    float vh[3], vl[3];  // compensated float velocity (delta form)
    double vd[3];        // float64 velocity (consistent form)
};

// B of the dipole (moment (0, 0, -|m|) at the origin), K = mu0/4pi |m|
D3 dipole64(const State& p, double K) {
    const double x = (double)p.hi[0] + p.lo[0], y = (double)p.hi[1] + p.lo[1], z = (double)p.hi[2] + p.lo[2];
    const double r2 = x * x + y * y + z * z, r = std::sqrt(r2);
    const double k3 = K / (r2 * r), mr = -z / r;
    return {k3 * (3.0 * mr * x / r), k3 * (3.0 * mr * y / r), k3 * (3.0 * mr * z / r + 1.0)};
}

F3 dipole32(const State& p, float Kf) {
    const F3 d{p.hi[0] + p.lo[0], p.hi[1] + p.lo[1], p.hi[2] + p.lo[2]};
    const float ir = (float)(1.0 / std::sqrt((double)dotf(d, d)));  // correctly rounded rsqrt, as __frsqrt_rn
    const F3 rh{ir * d.x, ir * d.y, ir * d.z};
    const float mr = -rh.z, k = Kf * ir * ir * ir;
    return {k * (3.0f * mr * rh.x), k * (3.0f * mr * rh.y), k * (3.0f * mr * rh.z + 1.0f)};
}

// closed-form rotation factors of MultistepBoris{4}(n = 2) from |t|^2 in float
void factors32(float s, float& c1m1, float& c2, float& c3, float& fN) {
    fN = 1.0f + s * (1.0f / 3.0f);
    s = fN * fN * s;
    float zr = 1.0f, q = 0.0f, A = 1.0f;
    for (int k = 0; k < 2; ++k) {
        const float nzr = zr - s * q;
        q = zr + q;
        zr = nzr;
        A = A * (1.0f + s);
    }
    const float invA = 1.0f / A;
    c2 = 2.0f * zr * q * invA;
    c3 = 2.0f * q * q * invA;
    c1m1 = -s * c3;
}

// one velocity update with factor fac = q2m dt / 4 (E = 0)
// field64: the field in float64 (else float32); consistent: float64
// velocity and the float factors made consistent in float64 (else the float
// delta form over a compensated float velocity)
void update(State& p, double fac, bool field64, bool consistent, double K, float Kf) {
    if (consistent) {
        D3 B;
        if (field64) {
            B = dipole64(p, K);
        } else {
            const F3 b = dipole32(p, Kf);
            B = {b.x, b.y, b.z};
        }
        D3 t{fac * B.x, fac * B.y, fac * B.z};
        float c1m1, c2, c3, fN;
        factors32((float)dotd(t, t), c1m1, c2, c3, fN);
        t = {fN * t.x, fN * t.y, fN * t.z};
        const double sd = dotd(t, t);
        double C1 = c1m1, C2 = c2, C3 = c3;
        const double hg = 0.5 * (C1 * (2.0 + C1) + C2 * C2 * sd);
        C1 -= hg * (1.0 + C1);
        C2 -= hg * C2;
        if (sd > 0.0) C3 -= (C1 + C3 * sd) / sd;
        const D3 v{p.vd[0], p.vd[1], p.vd[2]};
        const D3 vxt = crossd(v, t);
        const double vdt = dotd(v, t);
        p.vd[0] += C1 * v.x + C2 * vxt.x + C3 * vdt * t.x;
        p.vd[1] += C1 * v.y + C2 * vxt.y + C3 * vdt * t.y;
        p.vd[2] += C1 * v.z + C2 * vxt.z + C3 * vdt * t.z;
        return;
    }
    F3 B;
    if (field64) {
        const D3 b = dipole64(p, K);
        B = {(float)b.x, (float)b.y, (float)b.z};
    } else {
        B = dipole32(p, Kf);
    }
    const float f = (float)fac;
    F3 t{f * B.x, f * B.y, f * B.z};
    float c1m1, c2, c3, fN;
    factors32(dotf(t, t), c1m1, c2, c3, fN);
    t = {fN * t.x, fN * t.y, fN * t.z};
    const F3 v{p.vh[0], p.vh[1], p.vh[2]};
    const F3 vxt = crossf(v, t);
    const float vdt = dotf(v, t);
    cadd(p.vh[0], p.vl[0], c1m1 * v.x + c2 * vxt.x + (c3 * vdt) * t.x);
    cadd(p.vh[1], p.vl[1], c1m1 * v.y + c2 * vxt.y + (c3 * vdt) * t.y);
    cadd(p.vh[2], p.vl[2], c1m1 * v.z + c2 * vxt.z + (c3 * vdt) * t.z);
}

double vcomp(const State& p, int c, bool consistent) {
    return consistent ? p.vd[c] : (double)p.vh[c] + p.vl[c];
}

}  // namespace

// n particles, u0 (n x 6 row-major), per-particle dt and tend; final (x, v)
// into out (n x 6) and 1 (success) / 2 (left 1 - 15 R_E) into rc
extern "C" void fp32c_emulate(int64_t n, const double* u0, const double* dt_i, const double* tend_i, double q2m,
                              double K, double Re, int field64, int consistent, double* out, int8_t* rc) {
    const float Kf = (float)K;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        const double dt = dt_i[i];
        const int64_t nt = (int64_t)std::nearbyint(tend_i[i] / dt);
        State p;
        for (int c = 0; c < 3; ++c) {
            p.hi[c] = (float)u0[6 * i + c];
            p.lo[c] = (float)(u0[6 * i + c] - (double)p.hi[c]);
            const double v = u0[6 * i + 3 + c];
            p.vh[c] = (float)v;
            p.vl[c] = (float)(v - (double)p.vh[c]);
            p.vd[c] = v;
        }
        update(p, q2m * (-0.5 * dt) / 4.0, field64, consistent, K, Kf);
        int8_t r = 1;
        for (int64_t k = 0; k < nt; ++k) {
            State q = p;
            update(q, q2m * dt / 4.0, field64, consistent, K, Kf);
            for (int c = 0; c < 3; ++c) cadd(q.hi[c], q.lo[c], (float)(vcomp(q, c, consistent) * dt));
            const double x = (double)q.hi[0] + q.lo[0], y = (double)q.hi[1] + q.lo[1], z = (double)q.hi[2] + q.lo[2];
            const double rr = std::sqrt(x * x + y * y + z * z);
            if (rr < Re || rr > 15.0 * Re) {
                r = 2;
                break;
            }
            p = q;
        }
        update(p, q2m * (tend_i[i] - (nt - 0.5) * dt) / 4.0, field64, consistent, K, Kf);
        for (int c = 0; c < 3; ++c) {
            out[6 * i + c] = (double)p.hi[c] + p.lo[c];
            out[6 * i + 3 + c] = vcomp(p, c, consistent);
        }
        rc[i] = r;
    }
}
