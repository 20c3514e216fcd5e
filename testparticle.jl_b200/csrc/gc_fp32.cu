// gc_fp32.cu -- guiding-centre kernels with a float32 right-hand side
// (TP_GC_PREC_FP32RHS).  The state, the Runge-Kutta combinations, the
// embedded error norm and the step controller stay float64 (gc_common.cuh);
// get_gc_derivatives (src/equations.jl:329-360) is evaluated in float, with
// the field and its Jacobian in float.
#include "gc_common.cuh"

namespace tpb {

namespace {

struct V3f {
    float x, y, z;
};
__device__ __forceinline__ V3f operator+(V3f a, V3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3f operator-(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3f operator*(float s, V3f a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3f crossf(V3f a, V3f b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float dotf(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ V3f field32(const DevField& f, V3f r, float t) {
    switch (f.kind) {
        case TP_FIELD_UNIFORM:
            return {f.vf[0], f.vf[1], f.vf[2]};
        case TP_FIELD_AFFINE:
            return {f.vf[0] + f.Jf[0] * r.x + f.Jf[1] * r.y + f.Jf[2] * r.z + f.ratef[0] * t,
                    f.vf[1] + f.Jf[3] * r.x + f.Jf[4] * r.y + f.Jf[5] * r.z + f.ratef[1] * t,
                    f.vf[2] + f.Jf[6] * r.x + f.Jf[7] * r.y + f.Jf[8] * r.z + f.ratef[2] * t};
        case TP_FIELD_DIPOLE: {
            V3f d{r.x - f.cf[0], r.y - f.cf[1], r.z - f.cf[2]};
            V3f mh{f.mhatf[0], f.mhatf[1], f.mhatf[2]};
            float ir = rsqrtf(dotf(d, d));
            V3f rh = ir * d;
            float mr = dotf(mh, rh);
            float k3 = f.Kf * ir * ir * ir;  // coef |m| / r^3
            return {k3 * (3.0f * mr * rh.x - mh.x), k3 * (3.0f * mr * rh.y - mh.y), k3 * (3.0f * mr * rh.z - mh.z)};
        }
        default:
            return {0.0f, 0.0f, 0.0f};
    }
}

// B and its Jacobian in float (analytic kinds; grids through the float64 path)
__device__ __forceinline__ void field_jac32(const DevField& f, V3f r, float t, V3f& B, float J[9]) {
    for (int k = 0; k < 9; ++k) J[k] = 0.0f;
    if (f.kind == TP_FIELD_AFFINE) {
        B = field32(f, r, t);
        for (int k = 0; k < 9; ++k) J[k] = f.Jf[k];
        return;
    }
    if (f.kind == TP_FIELD_DIPOLE) {
        // unit-vector form: B = K/r^3 (3 (mh.rh) rh - mh),
        // dB_i/dx_j = K/r^4 (3 (mh_j rh_i + (mh.rh) delta_ij + mh_i rh_j) - 15 (mh.rh) rh_i rh_j)
        V3f d{r.x - f.cf[0], r.y - f.cf[1], r.z - f.cf[2]};
        float ir = rsqrtf(dotf(d, d));
        float rh[3] = {ir * d.x, ir * d.y, ir * d.z};
        float mh[3] = {f.mhatf[0], f.mhatf[1], f.mhatf[2]};
        float mr = mh[0] * rh[0] + mh[1] * rh[1] + mh[2] * rh[2];
        float k3 = f.Kf * ir * ir * ir;
        float k4 = k3 * ir;
        B = {k3 * (3.0f * mr * rh[0] - mh[0]), k3 * (3.0f * mr * rh[1] - mh[1]), k3 * (3.0f * mr * rh[2] - mh[2])};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                float dij = (i == j) ? mr : 0.0f;
                J[3 * i + j] = k4 * (3.0f * (mh[j] * rh[i] + dij + mh[i] * rh[j]) - 15.0f * mr * rh[i] * rh[j]);
            }
        return;
    }
    B = field32(f, r, t);
}

template <int GM>
struct RHS32 {
    static constexpr int kGM = GM;
    __device__ __forceinline__ G4 operator()(const DevFields& F, const G4& s, const GCPar& p,
                                             double t) const {
        V3f E, B;
        float J[9];
        V3f X{(float)s.y[0], (float)s.y[1], (float)s.y[2]};
        float tf = (float)t;
        if (GM != GM_ANALYTIC) {
            // grid fields: value and Jacobian from the float64 interpolant
            D3 Xd{s.y[0], s.y[1], s.y[2]};
            D3 Ed = field_eval64<GM == GM_ANY>(F.E, Xd, t), Bd;
            double Jd[9];
            field_jac64<GM>(F.B, Xd, t, Bd, Jd);
            E = {(float)Ed.x, (float)Ed.y, (float)Ed.z};
            B = {(float)Bd.x, (float)Bd.y, (float)Bd.z};
            for (int k = 0; k < 9; ++k) J[k] = (float)Jd[k];
        } else {
            E = field32(F.E, X, tf);
            field_jac32(F.B, X, tf, B, J);
        }
        float q2m = (float)p.q2m, upar = (float)s.y[3];
        float inv_B = rsqrtf(dotf(B, B));
        float Bmag = dotf(B, B) * inv_B;
        V3f bh = inv_B * B;
        V3f gB{J[0] * bh.x + J[3] * bh.y + J[6] * bh.z, J[1] * bh.x + J[4] * bh.y + J[7] * bh.z,
               J[2] * bh.x + J[5] * bh.y + J[8] * bh.z};
        V3f curlB{J[7] - J[5], J[2] - J[6], J[3] - J[1]};
        V3f curlb = inv_B * (curlB + crossf(bh, gB));
        (void)Bmag;
        V3f Bs = B + (upar / q2m) * curlb;
        V3f Es = E - (float)(p.mu / p.q) * gB;
        float inv_Bpar = 1.0f / dotf(bh, Bs);
        V3f v = inv_Bpar * (upar * Bs + crossf(Es, bh));
        float du = q2m * inv_Bpar * dotf(Bs, Es);
        return {{(double)v.x, (double)v.y, (double)v.z, (double)du}};
    }
};

}  // namespace

template <class R>
static const void* gc_kernel32(bool rk4, bool queue) {
    if (rk4) return queue ? (const void*)k_rk4<R, true> : (const void*)k_rk4<R, false>;
    return queue ? (const void*)k_rk45<R, true> : (const void*)k_rk45<R, false>;
}

const void* select_gc_kernel32(const GCArgs& a, bool queue) {
    const int gm = gc_grid_mode(a.f);
    bool rk4 = a.alg == TP_GC_RK4;
    if (gm == GM_ANY) return gc_kernel32<RHS32<GM_ANY>>(rk4, queue);
    return gm == GM_GRID ? gc_kernel32<RHS32<GM_GRID>>(rk4, queue) : gc_kernel32<RHS32<GM_ANALYTIC>>(rk4, queue);
}

cudaError_t launch_gc_fp32(const GCArgs& a, const LaunchCfg& c, cudaStream_t s) {
    const void* f = select_gc_kernel32(a, a.use_queue != 0);
    void* args[] = {const_cast<GCArgs*>(&a)};
    return cudaLaunchKernel(f, dim3(c.grid), dim3(c.block), args, 0, s);
}

}  // namespace tpb
