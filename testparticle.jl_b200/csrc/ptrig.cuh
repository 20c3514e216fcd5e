// ptrig.cuh -- portable sin / cos / atan2 in float64, shared by the float64
// kernels that must agree bit for bit with their CPU restatement: the
// gyrophase of the adaptive hybrid solver (hybrid.cu) and the closed-form
// rotation of MultistepBoris (multistep_rot64, fields64.cuh; the reference
// calls atan and sincos at src/boris/multistep_boris.jl:110-119).  Built from
// +, -, *, /, sqrt and rint only, so a translation unit compiled with
// -fmad=false gives the same bits as the CPU restatement compiled with
// -ffp-contract=off, whatever the platform's libm does.
#pragma once

namespace tpb {

// Portable sin / cos / atan2 for the gyrophase, built from +, -, *, / and
// sqrt only, so that the kernel and its CPU restatement agree bit for bit
// (the hybrid's step and mode decisions amplify last-bit differences):
//   sincos  Cody-Waite reduction by pi/2 (pi/2 split in three parts), then the
//           Taylor series of sin and cos on [-pi/4, pi/4] to degree 21 / 22
//   atan    for t in [0, 1]: up to two half-angle reductions tan(a/2) =
//           t / (1 + sqrt(1 + t^2)) to t <= tan(pi/16), then the Taylor
//           series to degree 29
__device__ __forceinline__ void psincos(double x, double& s, double& c) {
    const double P1 = 1.570796325802803, P2 = 9.920935791635221e-10, P3 = 5.170182981794105e-19;
    const double kf = rint(x * 0.6366197723675814);
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

__device__ __forceinline__ double patan01(double t) {
    // halve the angle (tan(a/2) = t / (1 + sqrt(1 + t^2))) until |u| <= tan(pi/16)
    double u = t, scale = 1.0;
    if (u > 0.19891236737965800) {
        u = u / (1.0 + sqrt(1.0 + u * u));
        scale = 2.0;
    }
    if (u > 0.19891236737965800) {
        u = u / (1.0 + sqrt(1.0 + u * u));
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

__device__ __forceinline__ double patan2(double y, double x) {
    if (x == 0.0 && y == 0.0) return 0.0;
    const double ax = fabs(x), ay = fabs(y);
    double a = (ay <= ax) ? patan01(ay / ax) : 1.5707963267948966 - patan01(ax / ay);
    if (x < 0.0) a = 3.141592653589793 - a;
    return (y < 0.0) ? -a : a;
}

}  // namespace tpb
