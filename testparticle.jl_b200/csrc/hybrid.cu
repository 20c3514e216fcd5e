// hybrid.cu -- the adaptive hybrid guiding-centre / full-orbit solver,
// float64.  Compiled with -fmad=false (see fields64.cuh): the same operation
// order as the CPU restatement, and the gyrophase trigonometry is the
// portable psincos / patan2 of ptrig.cuh, so both agree to the last bit.
//
// One thread per particle runs _hybrid_adaptive! (src/hybrid.jl:234-474):
//   GC mode  RK45 (update_dp5, src/gc/rk45_gc.jl:7-47) with the hybrid's own
//            step control (hybrid.jl:346-390) and a gyrophase carried along
//            for the full-orbit reconstruction (_gc_to_full, src/gc/gc.jl:128-154)
//   FO mode  Boris leapfrog with dt = 2 pi safety_fo / (|q2m| |B|) clamped to
//            [dtmin, dtmax] (_fo_dt, hybrid.jl:226-232)
//   every check_interval steps the adiabaticity (adiabaticity_components,
//   src/utility/utility.jl:554-577) decides the mode, with the hysteresis
//   thresholds threshold_gc_to_fo >= threshold_fo_to_gc.
#include "gc_common.cuh"

namespace tpb {

namespace {

constexpr double kTwoPi = 6.283185307179586;
constexpr double kTwoPiLo = 2.4492935982947064e-16;  // 2 pi - kTwoPi

// get_perp_vector (src/utility/utility.jl:119-126)
__device__ __forceinline__ void perp_vectors(D3 b, D3& e1, D3& e2) {
    D3 bh = b / norm(b);
    D3 v = fabs(bh.z) < 0.9 ? D3{0.0, 0.0, 1.0} : D3{0.0, 1.0, 0.0};
    D3 c = cross(v, bh);
    e1 = c / norm(c);
    e2 = cross(bh, e1);
}

// x reduced to [0, 2 pi) with 2 pi carried as two doubles (mod2pi)
__device__ __forceinline__ double mod2pi_d(double x) {
    double k = floor(x / kTwoPi);
    double r = fma(-k, kTwoPi, x);
    r = fma(-k, kTwoPiLo, r);
    if (r < 0.0) r = (r + kTwoPi) + kTwoPiLo;
    else if (r >= kTwoPi) r = (r - kTwoPi) - kTwoPiLo;
    return r;
}

// _get_gc_parameters (src/gc/gc.jl:13-39): X, v_par, mu, gyrophase
template <int GM>
__device__ __forceinline__ void gc_params(const DevFields& F, D3 x, D3 v, double q, double m, double t, D3& X,
                                          double& vpar, double& mu, double& phase) {
    D3 bp = field_val64<GM>(F.B, x, t);
    double Bmp = norm(bp);
    D3 bhp = bp / Bmp;
    D3 rho = cross(bhp, v) / (q / m * Bmp);
    X = x - rho;
    D3 b = field_val64<GM>(F.B, X, t);
    double Bmag = norm(b);
    D3 bh = b / Bmag;
    vpar = dot(bh, v);
    D3 vperp = v - vpar * bh;
    D3 e = field_val64<GM>(F.E, X, t);
    D3 vE = cross(e, bh) / Bmag;
    D3 w = vperp - vE;
    mu = m * dot(w, w) / (2.0 * Bmag);
    D3 e1, e2;
    perp_vectors(bh, e1, e2);
    phase = patan2(dot(w, e2), dot(w, e1));
}

// _gc_to_full (src/gc/gc.jl:128-154)
template <int GM>
__device__ __forceinline__ void gc_full(const DevFields& F, const G4& s, double q, double m, double mu, double t,
                                        double phase, D3& x, D3& v) {
    D3 R{s.y[0], s.y[1], s.y[2]};
    D3 E = field_val64<GM>(F.E, R, t), B = field_val64<GM>(F.B, R, t);
    double Bmag = norm(B);
    D3 bh = B / Bmag;
    D3 vE = cross(E, bh) / Bmag;
    double w = sqrt(2.0 * mu * Bmag / m);
    D3 e1, e2;
    perp_vectors(bh, e1, e2);
    double sp, cp;
    psincos(phase, sp, cp);
    D3 vperp = w * (cp * e1 + sp * e2) + vE;
    v = s.y[3] * bh + vperp;
    double Om = q * Bmag / m;
    x = R + cross(bh, vperp) / Om;
}

// adiabaticity_components (src/utility/utility.jl:554-577):
// (rho / R_c, rho / L_B, rho ||JB||_F / |B|)
template <int GM>
__device__ __forceinline__ void adia_components(const DevFields& F, D3 x, double q, double m, double mu, double t,
                                                double c[3]) {
    D3 B;
    double J[9];
    field_jac64<GM>(F.B, x, t, B, J);
    double Bmag = norm(B);
    if (Bmag == 0.0) {
        c[0] = c[1] = c[2] = __longlong_as_double(0x7ff0000000000000ULL);
        return;
    }
    double rho = sqrt(2.0 * mu * m / Bmag) / fabs(q);
    D3 bh = B / Bmag;
    D3 gB{(J[0] * bh.x + J[3] * bh.y) + J[6] * bh.z, (J[1] * bh.x + J[4] * bh.y) + J[7] * bh.z,
          (J[2] * bh.x + J[5] * bh.y) + J[8] * bh.z};
    double gBm = norm(gB);
    double LB = (gBm == 0.0) ? __longlong_as_double(0x7ff0000000000000ULL) : Bmag / gBm;
    c[1] = rho / LB;
    D3 Jb{(J[0] * bh.x + J[1] * bh.y) + J[2] * bh.z, (J[3] * bh.x + J[4] * bh.y) + J[5] * bh.z,
          (J[6] * bh.x + J[7] * bh.y) + J[8] * bh.z};
    D3 kap = (Jb + bh * (-dot(gB, bh))) / Bmag;
    c[0] = rho * norm(kap);
    // sum(abs2, JB) in Julia's column-major order
    double fro = J[0] * J[0];
    const int ord[8] = {3, 6, 1, 4, 7, 2, 5, 8};
    for (int k = 0; k < 8; ++k) fro = fro + J[ord[k]] * J[ord[k]];
    c[2] = rho * sqrt(fro) / Bmag;
}

// _adia_select (hybrid.jl:195-205)
__device__ __forceinline__ double adia_select(const double c[3], int mode) {
    if (mode == TP_ADIA_CURVATURE) return c[0];
    if (mode == TP_ADIA_GRADB) return c[1];
    if (mode == TP_ADIA_JACOBIAN) return c[2];
    if (isnan(c[0]) || isnan(c[1])) return c[0] + c[1];
    return c[0] < c[1] ? c[1] : c[0];
}

template <int GM>
__device__ __forceinline__ double fo_dt(const HybridArgs& a, D3 r, double t) {
    double Bmag = norm(field_val64<GM>(a.f.B, r, t));
    double om = fabs(a.q2m) * Bmag;
    double dt = kTwoPi * a.safety_fo / om;
    return dt > a.dtmax ? a.dtmax : (dt < a.dtmin ? a.dtmin : dt);
}

// update_velocity (src/boris/boris.jl:38-45) with the fields at (r, t)
template <int GM>
__device__ __forceinline__ D3 velocity(const HybridArgs& a, D3 v, D3 r, double dt, double t) {
    D3 E = field_val64<GM>(a.f.E, r, t), B = field_val64<GM>(a.f.B, r, t);
    return vel_update64<false>(v, E, B, a.q2m, dt, 2, 1);
}

__device__ __forceinline__ void save_state(const HybridArgs& a, int64_t i, int32_t k, D3 x, D3 v, double t) {
    if (k >= a.nslots) {
        set_status(a.status, TP_E_OVERFLOW);
        return;
    }
    const int64_t n = a.n;
    a.t_out[(int64_t)k * n + i] = t;
    double* u = a.u_out + ((int64_t)k * 6) * n + i;
    u[0] = x.x;
    u[n] = x.y;
    u[2 * n] = x.z;
    u[3 * n] = v.x;
    u[4 * n] = v.y;
    u[5 * n] = v.z;
}

__device__ __forceinline__ void save_adia(const HybridArgs& a, int64_t i, int32_t k, double t, double eps,
                                          bool gc) {
    if (!a.save_adia) return;
    if (k >= a.aslots) {
        set_status(a.status, TP_E_OVERFLOW);
        return;
    }
    const int64_t n = a.n;
    a.at_out[(int64_t)k * n + i] = t;
    a.av_out[((int64_t)k * 2) * n + i] = eps;
    a.av_out[((int64_t)k * 2 + 1) * n + i] = gc ? 0.0 : 1.0;
}

}  // namespace

template <int GM>
__global__ void __launch_bounds__(256, 1) k_hybrid(HybridArgs a) {
    const RHS64<GM> f;
    const bool is_td = !fields_static(a.f);
    const uint64_t t_start = globaltimer_ns();
    const double q = a.q2m * a.m;
    const double safety_gc = 0.9, max_growth = 5.0, min_growth = 0.2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double* u0 = a.u0 + 6 * i;
        D3 r{u0[0], u0[1], u0[2]}, v{u0[3], u0[4], u0[5]};
        double t = a.t0;
        GCPar p{q, a.q2m, 0.0};
        D3 X;
        double vpar, mu, phase;
        gc_params<GM>(a.f, r, v, q, a.m, t, X, vpar, mu, phase);
        double c[3];
        adia_components<GM>(a.f, r, q, a.m, mu, t, c);
        double eps = adia_select(c, a.adia_mode);
        // start in GC only when clearly adiabatic (hybrid.jl:257-279)
        bool gc = eps < a.th_gc_fo;
        G4 xg{{0.0, 0.0, 0.0, 0.0}};
        double dt;
        if (gc) {
            xg = {{X.x, X.y, X.z, vpar}};
            p.mu = mu;
            double Bmag = norm(field_val64<GM>(a.f.B, X, t));
            dt = 0.5 * kTwoPi / fabs(a.q2m * Bmag);
        } else {
            dt = fo_dt<GM>(a, r, t);
            v = velocity<GM>(a, v, r, -0.5 * dt, t);
        }
        int32_t na = 0, iout = 0;
        save_adia(a, i, na++, t, eps, gc);
        double t_last = t;
        if (a.save_start) {
            save_state(a, i, iout++, D3{u0[0], u0[1], u0[2]}, D3{u0[3], u0[4], u0[5]}, t);
        }
        int64_t steps = 0, it = 1, loops = 0;
        int ret = TP_RET_SUCCESS;
        while (t < a.t1 && steps < a.maxiters) {
            if ((++loops & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                set_status(a.status, TP_E_TIMEOUT);
                ret = TP_RET_DEFAULT;
                break;
            }
            if (gc) {
                if (it % a.check == 0) {
                    adia_components<GM>(a.f, D3{xg.y[0], xg.y[1], xg.y[2]}, q, a.m, mu, t, c);
                    eps = adia_select(c, a.adia_mode);
                    save_adia(a, i, na++, t, eps, true);
                    if (eps >= a.th_gc_fo) {  // GC -> FO
                        gc = false;
                        gc_full<GM>(a.f, xg, q, a.m, mu, t, phase, r, v);
                        dt = fo_dt<GM>(a, r, t);
                        v = velocity<GM>(a, v, r, -0.5 * dt, t);
                        continue;
                    }
                }
                if (t + dt > a.t1) dt = a.t1 - t;
                G4 dx, Er, y7, k7;
                update_dp5(f, a.f, xg, p, dt, t, f(a.f, xg, p, t), dx, Er, y7, k7);
                G4 yn = gadd(xg, dx);
                double sum_sq = 0.0;
                for (int k = 0; k < 4; ++k) {
                    double ax_ = fabs(xg.y[k]), ay_ = fabs(yn.y[k]);
                    double sc = a.abstol + ((ax_ < ay_) ? ay_ : ax_) * a.reltol;
                    double qk = Er.y[k] / sc;
                    sum_sq = sum_sq + qk * qk;
                }
                double er = 0.5 * sqrt(sum_sq);
                if (isnan(er)) {  // the reference would retry this step forever
                    ret = TP_RET_TERMINATED;
                    break;
                }
                if (er <= 1.0) {
                    if (a.term.flags && outside_gc(a.term, yn, t + dt)) break;
                    t += dt;
                    xg = yn;
                    double Bs = norm(field_val64<GM>(a.f.B, D3{xg.y[0], xg.y[1], xg.y[2]}, t));
                    phase = mod2pi_d(phase - dt * (a.q2m * Bs));
                    if (a.save_everystep && it % a.ssi == 0) {
                        D3 xs, vs;
                        gc_full<GM>(a.f, xg, q, a.m, mu, t, phase, xs, vs);
                        save_state(a, i, iout++, xs, vs, t);
                        t_last = t;
                    }
                    steps += 1;
                    it += 1;
                }
                double scale = (er == 0.0) ? max_growth : safety_gc * pow02_rn(1.0 / er);
                scale = (scale < max_growth) ? scale : max_growth;
                scale = (min_growth < scale) ? scale : min_growth;
                dt *= scale;
                if (dt < 1.0e-14) break;
            } else {
                if (it % a.check == 0) {
                    const double t_sync = is_td ? t : 0.0;
                    D3 vs = velocity<GM>(a, v, r, 0.5 * dt, t_sync);
                    D3 Xf;
                    double vparf, muf, phasef;
                    gc_params<GM>(a.f, r, vs, q, a.m, t, Xf, vparf, muf, phasef);
                    adia_components<GM>(a.f, Xf, q, a.m, muf, t, c);
                    eps = adia_select(c, a.adia_mode);
                    save_adia(a, i, na++, t, eps, false);
                    if (eps < a.th_fo_gc) {  // FO -> GC
                        gc = true;
                        xg = {{Xf.x, Xf.y, Xf.z, vparf}};
                        p.mu = muf;
                        mu = muf;
                        phase = phasef;
                        double Bmag = norm(field_val64<GM>(a.f.B, r, t));
                        dt = 0.5 * kTwoPi / fabs(a.q2m * Bmag);
                        continue;
                    }
                }
                if (t + dt > a.t1) dt = a.t1 - t;
                D3 vprev = v;
                v = velocity<GM>(a, v, r, dt, t + 0.5 * dt);
                D3 rn = r + v * dt;
                double tn = t + dt;
                if (a.term.flags && outside64(a.term, rn, v, tn)) break;
                if (a.save_everystep && it - 1 > 0 && (it - 1) % a.ssi == 0) {
                    D3 vsave = velocity<GM>(a, vprev, r, 0.5 * dt, t);
                    save_state(a, i, iout++, r, vsave, t);
                    t_last = t;
                }
                r = rn;
                t = tn;
                it += 1;
                steps += 1;
            }
        }
        // final save (hybrid.jl:449-459)
        if (a.save_end && (iout == 0 || t_last != t)) {
            if (gc) {
                D3 xs, vs;
                gc_full<GM>(a.f, xg, q, a.m, mu, t, phase, xs, vs);
                save_state(a, i, iout++, xs, vs, t);
            } else {
                const double t_final = is_td ? t : 0.0;
                save_state(a, i, iout++, r, velocity<GM>(a, v, r, 0.5 * dt, t_final), t);
            }
        }
        a.nsaved[i] = iout;
        if (a.save_adia) a.nadia[i] = na;
        a.retcode[i] = (int8_t)(ret != TP_RET_SUCCESS ? ret
                                                      : (steps >= a.maxiters ? TP_RET_MAXITERS : TP_RET_SUCCESS));
        a.nsteps[i] = steps;
    }
}

// gc_to_full (src/gc/gc.jl:106-154) at n guiding-centre states: the
// conversion of the hybrid solver, with the same portable sin / cos
template <int GM>
__global__ void k_gc_to_full(GCFullArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double* y = a.y + 4 * i;
    G4 s{{y[0], y[1], y[2], y[3]}};
    D3 x, v;
    gc_full<GM>(a.f, s, a.q, a.m, a.mu[i], a.t, a.phase_i ? a.phase_i[i] : a.phase, x, v);
    double* o = a.xv + 6 * i;
    o[0] = x.x;
    o[1] = x.y;
    o[2] = x.z;
    o[3] = v.x;
    o[4] = v.y;
    o[5] = v.z;
}

cudaError_t launch_gc_to_full(const GCFullArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    const int gm = gc_grid_mode(a.f);
    const void* k = gm == GM_ANY    ? (const void*)k_gc_to_full<GM_ANY>
                    : gm == GM_GRID ? (const void*)k_gc_to_full<GM_GRID>
                                    : (const void*)k_gc_to_full<GM_ANALYTIC>;
    const int block = 128;
    void* args[] = {const_cast<GCFullArgs*>(&a)};
    return cudaLaunchKernel(k, dim3((unsigned)((a.n + block - 1) / block)), dim3(block), args, 0, s);
}

static const void* hybrid_kernel(const HybridArgs& a) {
    const int gm = gc_grid_mode(a.f);
    return gm == GM_ANY ? (const void*)k_hybrid<GM_ANY>
                        : (gm == GM_GRID ? (const void*)k_hybrid<GM_GRID> : (const void*)k_hybrid<GM_ANALYTIC>);
}

cudaError_t prime_hybrid(const HybridArgs& a) {
    cudaFuncAttributes at;
    return cudaFuncGetAttributes(&at, hybrid_kernel(a));
}

cudaError_t launch_hybrid(const HybridArgs& a, int block, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    if (block <= 0) block = 128;
    int64_t grid = (a.n + block - 1) / block;
    void* args[] = {const_cast<HybridArgs*>(&a)};
    return cudaLaunchKernel(hybrid_kernel(a), dim3((unsigned)grid), dim3(block), args, 0, s);
}

}  // namespace tpb
