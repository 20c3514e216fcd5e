// gc_common.cuh -- guiding-centre RK4 / RK45 drivers, templated on the
// right-hand side.  The state, the Runge-Kutta combinations, the error norm
// and the step-size controller are float64 in every variant; the RHS
// (get_gc_derivatives, src/equations.jl:329-360) is float64 (RHS64, the
// drop-in) or float32 (RHS32).
//
//   k_rk4<RHS, QUEUE>   _rk4!  (src/gc/rk4_gc.jl:27-130)
//   k_rk45<RHS, QUEUE>  _rk45! (src/gc/rk45_gc.jl:52-173)
#pragma once

#include "fields64.cuh"
#include "tp_launch.h"

namespace tpb {

struct G4 {
    double y[4];
};
__device__ __forceinline__ G4 gadd(const G4& a, const G4& b) {
    return {{a.y[0] + b.y[0], a.y[1] + b.y[1], a.y[2] + b.y[2], a.y[3] + b.y[3]}};
}
__device__ __forceinline__ G4 gscale(double s, const G4& a) {
    return {{s * a.y[0], s * a.y[1], s * a.y[2], s * a.y[3]}};
}

struct GCPar {
    double q, q2m, mu;
};

// get_gc_derivatives (src/equations.jl:329-360), float64
// the grid mode a guiding-centre kernel is selected for
__host__ __device__ __forceinline__ int gc_grid_mode(const DevFields& f) {
    const bool ge = f.E.kind == TP_FIELD_GRID, gb = f.B.kind == TP_FIELD_GRID;
    if ((ge && f.E.general) || (gb && f.B.general)) return GM_ANY;
    if (f.E.kind == TP_FIELD_SERIES || f.B.kind == TP_FIELD_SERIES) return GM_ANY;
    const bool quad = f.E.kind == TP_FIELD_QUADRATIC || f.B.kind == TP_FIELD_QUADRATIC;
    return (ge || gb || quad) ? GM_GRID : GM_ANALYTIC;
}

template <int GM>
struct RHS64 {
    static constexpr int kGM = GM;
    __device__ __forceinline__ G4 operator()(const DevFields& F, const G4& s, const GCPar& p,
                                             double t) const {
        D3 X{s.y[0], s.y[1], s.y[2]};
        D3 E = field_val64<GM>(F.E, X, t);
        D3 B;
        double J[9];
        field_jac64<GM>(F.B, X, t, B, J);
        double Bmag = norm(B);
        D3 bh = B / Bmag;
        D3 gB{(J[0] * bh.x + J[3] * bh.y) + J[6] * bh.z, (J[1] * bh.x + J[4] * bh.y) + J[7] * bh.z,
              (J[2] * bh.x + J[5] * bh.y) + J[8] * bh.z};
        D3 curlB{J[7] - J[5], J[2] - J[6], J[3] - J[1]};
        D3 curlb = (curlB + cross(bh, gB)) / Bmag;
        D3 Bs = B + (s.y[3] / p.q2m) * curlb;
        D3 Es = E - (p.mu / p.q) * gB;
        double inv_Bpar = 1.0 / dot(bh, Bs);
        D3 v = (s.y[3] * Bs + cross(Es, bh)) * inv_Bpar;
        double du = dot((p.q2m * inv_Bpar) * Bs, Es);
        return {{v.x, v.y, v.z, du}};
    }
};

__device__ __forceinline__ bool outside_gc(const DevTerm& T, const G4& u, double t) {
    int f = T.flags;
    if (f & TP_TERM_NAN)
        for (int k = 0; k < 4; ++k)
            if (isnan(u.y[k])) return true;
    if (f & TP_TERM_SHELL) {
        double rr = sqrt((u.y[0] * u.y[0] + u.y[1] * u.y[1]) + u.y[2] * u.y[2]);
        if (rr < T.rmin || rr > T.rmax) return true;
    }
    if (f & TP_TERM_BOX)
        for (int c = 0; c < 3; ++c)
            if (u.y[c] < T.lo[c] || u.y[c] > T.hi[c]) return true;
    if (f & TP_TERM_TIME)
        if (t > T.tmax) return true;
    return false;
}

__device__ __forceinline__ GCPar gc_par(const GCArgs& a, int64_t i) {
    return {a.q_i ? a.q_i[i] : a.q, a.q2m_i ? a.q2m_i[i] : a.q2m, a.mu_i ? a.mu_i[i] : a.mu};
}

template <int GM>
struct GCSaver {
    const GCArgs& a;
    int W;
    __device__ GCSaver(const GCArgs& a_)
        : a(a_), W(4 + (a_.save_fields ? 6 : 0) + (a_.save_work ? 4 : 0)) {}
    // slot k: (X, v_par), then E and B when save_fields
    // (_prepare_saved_data_gc, src/gc/gc_solver.jl:233-248); the four
    // work-rate columns of save_work are filled by a post-pass
    __device__ __forceinline__ void save(int64_t i, int64_t k, const G4& s, double t) const {
        if (k >= a.nslots) {
            set_status(a.status, TP_E_OVERFLOW);
            return;
        }
        const int64_t n = a.n;
        a.t_out[k * n + i] = t;
        double* u = a.u_out + (k * W) * n + i;
        for (int c = 0; c < 4; ++c) u[c * n] = s.y[c];
        const D3 X{s.y[0], s.y[1], s.y[2]};
        if (a.save_fields) {
            D3 E = field_val64<GM>(a.f.E, X, t), B = field_val64<GM>(a.f.B, X, t);
            u[4 * n] = E.x;
            u[5 * n] = E.y;
            u[6 * n] = E.z;
            u[7 * n] = B.x;
            u[8 * n] = B.y;
            u[9 * n] = B.z;
        }
    }
};

template <bool QUEUE>
__device__ __forceinline__ int64_t gc_next(const GCArgs& a, int64_t& first) {
    if (!QUEUE) {
        int64_t g = first;
        first = a.n;
        return g;
    }
    return (int64_t)atomicAdd(a.queue, 1ULL);
}


// update_rk4, src/gc/rk4_gc.jl:7-22.  The stages run as a loop that is not
// unrolled (the right-hand side inlined once, as in update_dp5); the sum
// ((k1 + 2 k2) + 2 k3) + k4 is accumulated in the reference's order.
template <class RHS>
__device__ __forceinline__ G4 update_rk4(const RHS& f, const DevFields& F, const G4& y,
                                         const GCPar& p, double dt, double t) {
    G4 k = f(F, y, p, t);
    G4 sum = k;
#pragma unroll 1
    for (int st = 1; st < 4; ++st) {
        const double h = st < 3 ? 0.5 * dt : dt;
        G4 yt = gadd(y, gscale(h, k));
        k = f(F, yt, p, t + h);
        sum = st < 3 ? gadd(sum, gscale(2.0, k)) : gadd(sum, k);
    }
    return gscale(dt / 6.0, sum);
}

template <class RHS, bool QUEUE>
__global__ void __launch_bounds__(256) k_rk4(GCArgs a) {
    const RHS f;
    const GCSaver<RHS::kGM> S(a);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t i = -1, it = 0, iout = 0, nt = 0, nout = 0;
    G4 xv;
    GCPar p{0, 0, 0};
    double t_last = 0, dt = 0, t1 = 0;
    bool timed_out = false;
    for (;;) {
        if (i < 0) {
            i = gc_next<QUEUE>(a, first);
            if (i >= a.n) break;
            p = gc_par(a, i);
            const double* y0 = a.y0 + 4 * i;
            xv = {{y0[0], y0[1], y0[2], y0[3]}};
            dt = a.dt_i ? a.dt_i[i] : a.dt;
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            if (a.dt_i || a.tend_i) {
                // _prepare_gc (gc_solver.jl:198-225) for this particle
                nt = jl_round((t1 - a.t0) / dt);
                if (nt > a.maxiters) nt = a.maxiters;
                nout = (a.save_start ? 1 : 0);
                if (a.save_everystep) {
                    int64_t st = nt / a.ssi;
                    bool last_is_step = (nt > 0) && (nt % a.ssi == 0);
                    nout += st;
                    if (!a.save_end && last_is_step) nout -= 1;
                    if (a.save_end && !last_is_step) nout += 1;
                } else if (a.save_end) {
                    nout += 1;
                }
            } else {
                nt = a.nt;
                nout = a.nout;
            }
            iout = 0;
            if (a.save_start) {
                S.save(i, 0, xv, a.t0);
                t_last = a.t0;
                iout = 1;
            }
            it = 1;
            timed_out = false;
        }
        bool done = !(it <= nt && it <= a.maxiters);
        if (!done) {
            double t = fma((double)(it - 1), dt, a.t0);
            G4 dx = update_rk4(f, a.f, xv, p, dt, t);
            G4 xn = gadd(xv, dx);
            if (a.term.flags && outside_gc(a.term, xn, t + dt)) {
                done = true;
            } else {
                xv = xn;
                if (a.save_everystep && (it % a.ssi == 0)) {
                    iout += 1;
                    if (iout <= nout) {
                        S.save(i, iout - 1, xv, t + dt);
                        t_last = t + dt;
                    }
                }
                it += 1;
                done = !(it <= nt && it <= a.maxiters);
                if ((it & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                    set_status(a.status, TP_E_TIMEOUT);
                    timed_out = true;
                    done = true;
                }
            }
        }
        if (done) {
            int64_t final_step = it - 1;
            bool sf = a.save_end || (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
            if (iout < nout && sf) {
                double t_final = (final_step == nt) ? t1 : fma((double)final_step, dt, a.t0);
                if (iout == 0 || t_last < t_final) {
                    S.save(i, iout, xv, t_final);
                    iout += 1;
                }
            }
            int ret;
            if (timed_out)
                ret = TP_RET_DEFAULT;
            else if (it <= nt && it <= a.maxiters)
                ret = TP_RET_TERMINATED;
            else if (it > a.maxiters)
                ret = TP_RET_MAXITERS;
            else
                ret = TP_RET_SUCCESS;
            a.nsaved[i] = (int32_t)iout;
            a.retcode[i] = (int8_t)ret;
            a.nsteps[i] = final_step;
            i = -1;
        }
    }
}

// x^0.2 rounded to nearest: the step-size factor (1.0 / error_ratio)^0.2 of
// rk45_gc.jl:151.  CUDA's pow is accurate to 2 ulp, and a one-ulp change of
// the factor moves every later step, so the factor is refined to the
// correctly rounded value, which is also what the oracle computes: one
// Newton step for the real fifth root from z0 = pow(x, 0.2), with the
// residual z0^5 - x in double-double arithmetic (Dekker's exact product by
// fma; z0^5 - x is exact by Sterbenz's lemma), then the exponent correction
// x^(0.2 - 1/5) = 1 + d ln x for the float64 constant 0.2 = 1/5 + d,
// d = 2^-54 / 5.  Explicit _rn operations keep the sequence free of
// contraction in every translation unit.  Outside [1e-30, 1e30], where the
// controller clamps the factor anyway, z0 is returned.
__device__ __forceinline__ double pow02_rn(double x) {
    double z0 = pow(x, 0.2);
    if (!(x >= 1.0e-30 && x <= 1.0e30) || !(z0 > 0.0) || isinf(z0)) return z0;
    double a = __dmul_rn(z0, z0);
    double ae = fma(z0, z0, -a);
    double b = __dmul_rn(a, a);
    double be = __dadd_rn(fma(a, a, -b), __dmul_rn(__dmul_rn(2.0, a), ae));
    double c = __dmul_rn(b, z0);
    double ce = __dadd_rn(fma(b, z0, -c), __dmul_rn(be, z0));
    double r = __dadd_rn(__dsub_rn(c, x), ce);
    double corr = __ddiv_rn(-r, __dmul_rn(5.0, b));
    double t = __dmul_rn(0.2 * 0x1p-54, log(x));
    return __dadd_rn(z0, __dadd_rn(corr, __dmul_rn(z0, t)));
}

// update_dp5, src/gc/rk45_gc.jl:7-47 (tableau of rk45_gc.jl:9-20), with k1 =
// f(y, t) given by the caller; returns the seventh stage's input y7 and k7
// = f(y7, t + dt).  The stages run as a loop that is not unrolled, so the
// right-hand side is inlined once: seven inlined copies overflowed the
// instruction cache (the kernel stalled on instruction fetch).  Each stage's
// sum adds a_s1 k1 + a_s2 k2 + ... left to right, the reference's order, and
// its time is fma(c_s, dt, t) (c6 = c7 = 1: t + dt exactly).
struct DP5Tableau {
    double a[7][6];
    double c[7];
};
__constant__ const DP5Tableau kDP5 = {
    {{0, 0, 0, 0, 0, 0},
     {1.0 / 5, 0, 0, 0, 0, 0},
     {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
     {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
     {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
     {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
     {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}},
    {0.0, 1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1.0, 1.0}};

template <class RHS>
__device__ __forceinline__ void update_dp5(const RHS& f, const DevFields& F, const G4& y,
                                           const GCPar& p, double dt, double t, const G4& k1, G4& dy, G4& err,
                                           G4& y7, G4& k7) {
    const double b1 = 35.0 / 384, b3 = 500.0 / 1113, b4 = 125.0 / 192, b5 = -2187.0 / 6784,
                 b6 = 11.0 / 84;
    const double e1 = 71.0 / 57600, e3 = -71.0 / 16695, e4 = 71.0 / 1920, e5 = -17253.0 / 339200,
                 e6 = 22.0 / 525, e7 = -1.0 / 40;
    G4 k[7];
    k[0] = k1;
    G4 yt;
#pragma unroll 1
    for (int st = 1; st < 7; ++st) {
        G4 acc = gscale(kDP5.a[st][0], k[0]);
        for (int j = 1; j < st; ++j) acc = gadd(acc, gscale(kDP5.a[st][j], k[j]));
        yt = gadd(y, gscale(dt, acc));
        k[st] = f(F, yt, p, fma(kDP5.c[st], dt, t));
    }
    y7 = yt;
    k7 = k[6];
    dy = gscale(dt, gadd(gadd(gadd(gadd(gscale(b1, k[0]), gscale(b3, k[2])), gscale(b4, k[3])),
                              gscale(b5, k[4])),
                         gscale(b6, k[5])));
    err = gscale(dt, gadd(gadd(gadd(gadd(gadd(gscale(e1, k[0]), gscale(e3, k[2])), gscale(e4, k[3])),
                                    gscale(e5, k[4])),
                               gscale(e6, k[5])),
                          gscale(e7, k[6])));
}

// Register cap 168 (65536 / 384): three blocks of 128 threads per SM for the
// float64 right-hand side instead of two, for a few bytes of spill.
template <class RHS, bool QUEUE>
__global__ void __launch_bounds__(384, 1) k_rk45(GCArgs a) {
    const RHS f;
    const GCSaver<RHS::kGM> S(a);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double safety = 0.9, max_growth = 5.0, min_growth = 0.2;
    int64_t i = -1, iout = 0, steps = 0, attempts = 0;
    G4 xv, k1;
    bool have_k1 = false;
    GCPar p{0, 0, 0};
    double t = 0, dt = 0, t_last = 0, t1 = 0;
    int ret = TP_RET_SUCCESS;
    for (;;) {
        if (i < 0) {
            i = gc_next<QUEUE>(a, first);
            if (i >= a.n) break;
            p = gc_par(a, i);
            const double* y0 = a.y0 + 4 * i;
            xv = {{y0[0], y0[1], y0[2], y0[3]}};
            t = a.t0;
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            if (a.dt_i) {
                dt = a.dt_i[i];
            } else if (!a.dt_given) {
                D3 R{xv.y[0], xv.y[1], xv.y[2]};
                double Bmag = norm(field_val64<RHS::kGM>(a.f.B, R, t));
                if (Bmag == 0.0 || p.q2m == 0.0) {
                    dt = 1.0e-6;
                } else {
                    double omega = fabs(p.q2m * Bmag);
                    dt = 0.5 * 6.283185307179586 / omega;
                }
            } else {
                dt = a.dt;
            }
            iout = 0;
            if (a.save_start) {
                S.save(i, 0, xv, t);
                t_last = t;
                iout = 1;
            }
            steps = 0;
            attempts = 0;
            ret = TP_RET_SUCCESS;
            have_k1 = false;
        }
        bool done = !(t < t1 && steps < a.maxiters);
        if (!done) {
            if (t + dt > t1) dt = t1 - t;
            // k1 = f(x, t) is the last attempt's k1 after a rejection (same x
            // and t) and its k7 after an acceptance whose seventh-stage input
            // equals the new state bit for bit (k7 is then f(x_new, t + dt)):
            // the same value the reference recomputes, one evaluation fewer
            if (!have_k1) k1 = f(a.f, xv, p, t);
            G4 dx, E, y7, k7;
            update_dp5(f, a.f, xv, p, dt, t, k1, dx, E, y7, k7);
            G4 yn = gadd(xv, dx);
            have_k1 = true;
            double sum_sq = 0.0;
            for (int k = 0; k < 4; ++k) {
                double ax_ = fabs(xv.y[k]), ay_ = fabs(yn.y[k]);
                double sc = fma((ax_ < ay_) ? ay_ : ax_, a.reltol, a.abstol);
                double qk = E.y[k] / sc;
                sum_sq = fma(qk, qk, sum_sq);
            }
            double error_ratio = 0.5 * sqrt(sum_sq);
            bool stop = false;
            // accept unless the ratio exceeds 1: a NaN ratio is accepted, as the
            // reference's @fastmath comparison does (the NaN state then ends
            // the trajectory through isoutside)
            if (!(error_ratio > 1.0)) {
                if (a.term.flags && outside_gc(a.term, yn, t + dt)) {
                    ret = TP_RET_TERMINATED;
                    stop = true;
                } else {
                    t += dt;
                    bool same = true;
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        same = same && __double_as_longlong(y7.y[k]) == __double_as_longlong(yn.y[k]);
                    if (same) k1 = k7;
                    have_k1 = same;
                    xv = yn;
                    if (a.save_everystep) {
                        S.save(i, iout, xv, t);
                        t_last = t;
                        iout += 1;
                    }
                    steps += 1;
                }
            }
            if (!stop) {
                double scale = (error_ratio == 0.0) ? max_growth : safety * pow02_rn(1.0 / error_ratio);
                scale = (max_growth < scale) ? max_growth : scale;
                scale = (min_growth < scale) ? scale : min_growth;
                dt *= scale;
                if (dt < 1.0e-14) stop = true;
            }
            attempts += 1;
            if ((attempts & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                set_status(a.status, TP_E_TIMEOUT);
                ret = TP_RET_DEFAULT;
                stop = true;
            }
            done = stop || !(t < t1 && steps < a.maxiters);
        }
        if (done) {
            if (a.save_end && (iout == 0 || t_last != t)) {
                S.save(i, iout, xv, t);
                iout += 1;
            }
            a.nsaved[i] = (int32_t)iout;
            a.retcode[i] = (int8_t)ret;
            a.nsteps[i] = steps;
            i = -1;
        }
    }
}

}  // namespace tpb
