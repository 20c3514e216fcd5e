// boris_fp32c.cu -- float32 push with compensated positions (TP_PREC_FP32C).
//
// Same algorithms and save semantics as boris_fp64.cu, with:
//  * positions as unevaluated float pairs (hi, lo): every update x += v*dt is
//    Knuth's TwoSum of hi and the increment followed by Dekker's Fast2Sum
//    renormalisation, so the position carries ~48 significant bits;
//  * on axes where every field is a periodic grid (and no spatial
//    termination predicate is set) hi is kept inside [x0, x0 + L) with an
//    integer wrap count, so the cell fraction is computed from a small
//    number and stays exact to ~1e-8 cells even for drifting particles;
//  * E, B, velocity and the rotation factors in float (rotation with correctly
//    rounded division, no approximate reciprocals);
//  * MultistepBoris in closed form without atan/sincos: with tau = |t_n|,
//    (1 + i tau)^n = zr + i tau q gives cos/sin of n*atan(tau), and the
//    coefficients of multistep_boris.jl:116-119 become
//      c1 = (zr^2 - tau^2 q^2)/A, c2 = 2 zr q / A, c3 = 2 q^2 / A, c6 = 2 R / A
//    with A = (1 + tau^2)^n and R = (n A - zr q) / tau^2 built by the
//    recurrence R_{k+1} = R_k + (k+1) A_k + 2 q_k^2 + zr_k q_k, which is free
//    of the cancellation the Taylor branch (multistep_boris.jl:99-108) guards;
//  * time t, the adaptive step dt = C/|B| and the end-of-span clipping in
//    float64 so that step decisions follow the float64 controller.
#include "fp32c_common.cuh"
#include "tp_device.cuh"
#include "tp_launch.h"

namespace tpb {

namespace {

template <int FK>
__device__ __forceinline__ bool outside32(const BorisArgs& a, const CPos& p, const typename Vel32<FK>::V& v,
                                          double t) {
    const DevTerm& T = a.term;
    int f = T.flags;
    if (f & TP_TERM_NAN)
        if (isnan(p.hi[0]) || isnan(p.hi[1]) || isnan(p.hi[2]) || Vel32<FK>::has_nan(v)) return true;
    if (f & (TP_TERM_SHELL | TP_TERM_BOX)) {
        // in float on hi + lo: no axis wraps when a spatial predicate is set,
        // and the float-side position already differs from the float64 one
        // by more than the float rounding of the test (no float64 sqrt)
        const float x = p.hi[0] + p.lo[0], y = p.hi[1] + p.lo[1], z = p.hi[2] + p.lo[2];
        if (f & TP_TERM_SHELL) {
            const float r2 = fmaf(x, x, fmaf(y, y, z * z));
            const float rmin2 = T.rmin > 0.0 ? (float)(T.rmin * T.rmin) : -1.0f;
            const float rmax2 = T.rmax >= 0.0 ? (float)(T.rmax * T.rmax) : -1.0f;
            if (r2 < rmin2 || r2 > rmax2) return true;
        }
        if (f & TP_TERM_BOX) {
            if (x < (float)T.lo[0] || x > (float)T.hi[0] || y < (float)T.lo[1] || y > (float)T.hi[1] ||
                z < (float)T.lo[2] || z > (float)T.hi[2])
                return true;
        }
    }
    if (f & TP_TERM_TIME)
        if (t > T.tmax) return true;
    return false;
}

template <int FK>
struct Saver32 {
    using P = Vel32<FK>;
    const BorisArgs& a;
    int W;
    // slot width: the state, E and B (float evaluation, as the push sees
    // them) when save_fields, and four work-rate columns when save_work that
    // a post-pass over the saved states fills (keeps that float64 code out
    // of this kernel's registers)
    __device__ Saver32(const BorisArgs& a_)
        : a(a_), W(6 + (a_.save_fields ? 6 : 0) + (a_.save_work ? 4 : 0)) {}
    __device__ __forceinline__ void save(int64_t i, int64_t k, const CPos& p, const typename P::V& v,
                                         double t) const {
        if (k >= a.nslots) {
            set_status(a.status, TP_E_OVERFLOW);
            return;
        }
        const int64_t n = a.n;
        a.t_out[k * n + i] = t;
        double* u = a.u_out + (k * W) * n + i;
        u[0 * n] = cpos_value(a, p, 0);
        u[1 * n] = cpos_value(a, p, 1);
        u[2 * n] = cpos_value(a, p, 2);
        u[3 * n] = P::comp(v, 0);
        u[4 * n] = P::comp(v, 1);
        u[5 * n] = P::comp(v, 2);
        if (a.save_fields) {
            typename P::Fv E, B;
            P::fields(a.f, p, t, E, B);
            u[6 * n] = E.x;
            u[7 * n] = E.y;
            u[8 * n] = E.z;
            u[9 * n] = B.x;
            u[10 * n] = B.y;
            u[11 * n] = B.z;
        }
    }
};

template <bool QUEUE>
__device__ __forceinline__ int64_t next_particle32(const BorisArgs& a, int64_t& first) {
    if (!QUEUE) {
        int64_t g = first;
        first = a.n;
        return take_particle(a, g);
    }
    return take_particle(a, (int64_t)atomicAdd(a.queue, 1ULL));
}

}  // namespace

// ---------------------------------------------------------------- fixed step
template <bool MULTI, bool QUEUE, int FK>
__global__ void __launch_bounds__(TPB_FIXED_BOUND(FK), 1) k_fixed32c(BorisArgs a) {
    using P = Vel32<FK>;
    using V = typename P::V;
    using Fv = typename P::Fv;
    const Saver32<FK> S(a);
    const bool stat = fields_static32(a.f);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;

    int64_t i = -1;
    CPos p;
    V v{};
    double dt = 0, t = 0, t1 = 0, t_last = 0;
    float dth = 0, dtl = 0;
    typename P::H hstep = 0;
    int64_t it = 0, nt = 0;
    int32_t nout = 0, iout = 0, csave = 0;

    for (;;) {
        if (i < 0) {
            i = next_particle32<QUEUE>(a, first);
            if (i >= a.n) break;
            dt = a.dt_i ? a.dt_i[i] : a.dt;
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            nt = (fabs(dt) < 10.0 * 2.220446049250313e-16) ? -1 : jl_round((t1 - a.t0) / dt);
            if (nt < 0 && fabs(dt) >= 10.0 * 2.220446049250313e-16) nt = -nt;
            if (nt < 0 || nt > a.maxiters) {
                set_status(a.status, TP_E_ARG);
                a.nsaved[i] = 0;
                a.retcode[i] = TP_RET_DEFAULT;
                a.nsteps[i] = 0;
                particle_done(a, i);
                i = -1;
                continue;
            }
            dth = (float)dt;
            dtl = (float)(dt - (double)dth);
            hstep = P::template fac<MULTI>(a, dt);
            nout = (int32_t)calc_nout(nt, a.ssi, a.save_start, a.save_end, a.save_everystep);
            const double* u0 = a.u0 + 6 * i;
            cpos_init(a, p, u0);
            v = P::init(u0 + 3);
            iout = 0;
            if (a.save_start) {
                a.t_out[i] = a.t0;  // save_start writes u0 exactly (slot 0)
                if (a.nslots > 0) {
                    double* u = a.u_out + i;
                    for (int c = 0; c < 6; ++c) u[c * a.n] = u0[c];
                    if (a.save_fields) {
                        Fv E, B;
                        P::fields(a.f, p, a.t0, E, B);
                        u[6 * a.n] = E.x; u[7 * a.n] = E.y; u[8 * a.n] = E.z;
                        u[9 * a.n] = B.x; u[10 * a.n] = B.y; u[11 * a.n] = B.z;
                    }
                } else {
                    set_status(a.status, TP_E_OVERFLOW);
                }
                t_last = a.t0;
                iout = 1;
            }
            Fv E, B;
            P::fields(a.f, p, a.t0, E, B);
            v = P::template step<MULTI>(v, E, B, a, -0.5 * dt);
            it = 1;
            t = a.t0 - 0.5 * dt;
            csave = 0;
        }

        bool done = it > nt;
        if (!done) {
            // v is v_{it-1/2} until the step is accepted: the save of r_{it-1}
            // and the termination rollback (the reference returns v_prev,
            // boris.jl:460) both use it, so no copy of it is kept
            t += dt;
            Fv E, B;
            P::fields(a.f, p, t, E, B);
            V vn = P::template step_h<MULTI>(v, E, B, a, hstep);
            CPos pn = p;
            P::push(a, pn, vn, dth, dtl, dt);
            if (a.term.flags && outside32<FK>(a, pn, vn, t + 0.5 * dt)) {
                done = true;
            } else {
                if (a.save_everystep && it > 1 && csave == 0) {
                    iout += 1;
                    if (iout <= nout) {
                        double t_cur = t - 0.5 * dt;
                        if (!stat) P::fields(a.f, p, t_cur, E, B);
                        V vs = P::template step<MULTI>(v, E, B, a, 0.5 * dt);
                        S.save(i, iout - 1, p, vs, t_cur);
                        t_last = t_cur;
                    }
                }
                p = pn;
                v = vn;
                it += 1;
                csave += 1;
                if (csave == a.ssi) csave = 0;
                done = it > nt;
                if ((it & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                    set_status(a.status, TP_E_TIMEOUT);
                    done = true;
                }
            }
        }
        if (done) {
            int64_t final_step = it - 1;
            bool save_final = a.save_end ||
                              (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
            if (iout < nout && save_final) {
                double t_final = (final_step == nt) ? t1 : fma((double)final_step, dt, a.t0);
                if (iout == 0 || t_last < t_final) {
                    double dt_final = t_final - fma((double)final_step - 0.5, dt, a.t0);
                    Fv E, B;
                    P::fields(a.f, p, t_final, E, B);
                    V vf = P::template step<MULTI>(v, E, B, a, dt_final);
                    S.save(i, iout, p, vf, t_final);
                    iout += 1;
                }
            }
            a.nsaved[i] = (int32_t)iout;
            a.retcode[i] = (int8_t)((iout < nout) ? TP_RET_TERMINATED : TP_RET_SUCCESS);
            a.nsteps[i] = final_step;
            particle_done(a, i);
            i = -1;
        }
    }
}

// ---------------------------------------------------------------- fixed step, several particles per thread
// PPT particles per thread ("slots"), advanced in lock step: each loop
// iteration first refills idle slots, then computes every slot's step (field,
// velocity update, push) as one straight-line block -- independent work the
// scheduler can interleave -- and then commits each slot (termination, saves,
// end of trajectory).  A slot without a particle computes on its stale state
// and commits nothing.  Static schedule: slot k of global thread g owns
// particle g + k * (threads in the grid).
template <bool MULTI, bool QUEUE, int FK, int PPT>
__global__ void __launch_bounds__(TPB_MAXT(FK) / PPT, 1) k_fixed32c_slots(BorisArgs a) {
    using P = Vel32<FK>;
    using V = typename P::V;
    using Fv = typename P::Fv;
    const Saver32<FK> S(a);
    const uint64_t t_start = globaltimer_ns();
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;

    int64_t first[PPT], i[PPT];
    CPos p[PPT];
    V v[PPT];
    double dt[PPT], t[PPT], t1[PPT], t_last[PPT];
    float dth[PPT], dtl[PPT];
    typename P::H hstep[PPT];
    int64_t it[PPT], nt[PPT];
    int32_t nout[PPT], iout[PPT], csave[PPT];
    bool dead[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        first[k] = g + k * gstride;
        i[k] = -1;
        dead[k] = false;
        v[k] = V{};
        dt[k] = t[k] = t1[k] = t_last[k] = 0.0;
        dth[k] = dtl[k] = 0.0f;
        hstep[k] = 0;
        it[k] = nt[k] = 0;
        nout[k] = iout[k] = csave[k] = 0;
        for (int c = 0; c < 3; ++c) {
            p[k].hi[c] = p[k].lo[c] = 0.0f;
            p[k].w[c] = 0;
        }
    }

    for (;;) {
        // ---- refill idle slots (_boris_single set-up, boris.jl:480-514)
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            while (!dead[k] && i[k] < 0) {
                i[k] = next_particle32<QUEUE>(a, first[k]);
                if (i[k] >= a.n) {
                    dead[k] = true;
                    break;
                }
                const int64_t ii = i[k];
                dt[k] = a.dt_i ? a.dt_i[ii] : a.dt;
                t1[k] = a.tend_i ? a.tend_i[ii] : a.t1;
                nt[k] = (fabs(dt[k]) < 10.0 * 2.220446049250313e-16) ? -1 : jl_round((t1[k] - a.t0) / dt[k]);
                if (nt[k] < 0 && fabs(dt[k]) >= 10.0 * 2.220446049250313e-16) nt[k] = -nt[k];
                if (nt[k] < 0 || nt[k] > a.maxiters) {
                    set_status(a.status, TP_E_ARG);
                    a.nsaved[ii] = 0;
                    a.retcode[ii] = TP_RET_DEFAULT;
                    a.nsteps[ii] = 0;
                    particle_done(a, ii);
                    i[k] = -1;
                    continue;
                }
                dth[k] = (float)dt[k];
                dtl[k] = (float)(dt[k] - (double)dth[k]);
                hstep[k] = P::template fac<MULTI>(a, dt[k]);
                nout[k] = (int32_t)calc_nout(nt[k], a.ssi, a.save_start, a.save_end, a.save_everystep);
                const double* u0 = a.u0 + 6 * ii;
                cpos_init(a, p[k], u0);
                v[k] = P::init(u0 + 3);
                iout[k] = 0;
                if (a.save_start) {
                    a.t_out[ii] = a.t0;  // save_start writes u0 exactly (slot 0)
                    if (a.nslots > 0) {
                        double* u = a.u_out + ii;
                        for (int c = 0; c < 6; ++c) u[c * a.n] = u0[c];
                        if (a.save_fields) {
                            Fv E, B;
                            P::fields(a.f, p[k], a.t0, E, B);
                            u[6 * a.n] = E.x; u[7 * a.n] = E.y; u[8 * a.n] = E.z;
                            u[9 * a.n] = B.x; u[10 * a.n] = B.y; u[11 * a.n] = B.z;
                        }
                    } else {
                        set_status(a.status, TP_E_OVERFLOW);
                    }
                    t_last[k] = a.t0;
                    iout[k] = 1;
                }
                Fv E, B;
                P::fields(a.f, p[k], a.t0, E, B);
                v[k] = P::template step<MULTI>(v[k], E, B, a, -0.5 * dt[k]);
                it[k] = 1;
                t[k] = a.t0 - 0.5 * dt[k];
                csave[k] = 0;
            }
        }
        bool any = false;
#pragma unroll
        for (int k = 0; k < PPT; ++k) any = any || !dead[k];
        if (!any) break;

        // ---- one step of every slot: field, velocity update, push.  v stays
        // v_{it-1/2} until the step is accepted: the save of r_{it-1} and the
        // termination rollback (the reference returns v_prev, boris.jl:460)
        // both use it
        V vn[PPT];
        CPos pn[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            Fv E, B;
            P::fields(a.f, p[k], t[k] + dt[k], E, B);
            vn[k] = P::template step_h<MULTI>(v[k], E, B, a, hstep[k]);
            pn[k] = p[k];
            P::push(a, pn[k], vn[k], dth[k], dtl[k], dt[k]);
        }

        // ---- commit (_boris_loop!, boris.jl:452-476), end of trajectory (:522-551)
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            if (dead[k]) continue;
            const int64_t ii = i[k];
            bool done = it[k] > nt[k];
            if (!done) {
                t[k] += dt[k];
                if (a.term.flags && outside32<FK>(a, pn[k], vn[k], t[k] + 0.5 * dt[k])) {
                    done = true;
                } else {
                    if (a.save_everystep && it[k] > 1 && csave[k] == 0) {
                        iout[k] += 1;
                        if (iout[k] <= nout[k]) {
                            const double t_cur = t[k] - 0.5 * dt[k];
                            Fv E, B;
                            P::fields(a.f, p[k], t_cur, E, B);
                            V vs = P::template step<MULTI>(v[k], E, B, a, 0.5 * dt[k]);
                            S.save(ii, iout[k] - 1, p[k], vs, t_cur);
                            t_last[k] = t_cur;
                        }
                    }
                    p[k] = pn[k];
                    v[k] = vn[k];
                    it[k] += 1;
                    csave[k] += 1;
                    if (csave[k] == a.ssi) csave[k] = 0;
                    done = it[k] > nt[k];
                    if ((it[k] & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                        set_status(a.status, TP_E_TIMEOUT);
                        done = true;
                    }
                }
            }
            if (done) {
                const int64_t final_step = it[k] - 1;
                const bool save_final = a.save_end ||
                                        (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
                if (iout[k] < nout[k] && save_final) {
                    const double t_final = (final_step == nt[k]) ? t1[k] : fma((double)final_step, dt[k], a.t0);
                    if (iout[k] == 0 || t_last[k] < t_final) {
                        const double dt_final = t_final - fma((double)final_step - 0.5, dt[k], a.t0);
                        Fv E, B;
                        P::fields(a.f, p[k], t_final, E, B);
                        V vf = P::template step<MULTI>(v[k], E, B, a, dt_final);
                        S.save(ii, iout[k], p[k], vf, t_final);
                        iout[k] += 1;
                    }
                }
                a.nsaved[ii] = (int32_t)iout[k];
                a.retcode[ii] = (int8_t)((iout[k] < nout[k]) ? TP_RET_TERMINATED : TP_RET_SUCCESS);
                a.nsteps[ii] = final_step;
                particle_done(a, ii);
                i[k] = -1;
            }
        }
    }
}

// ---------------------------------------------------------------- cubic grids, warp-cooperative
// E and B on one periodic, uniform, Cartesian 3-D grid interpolated at order
// 3 (cardinal_interp, src/utility/interpolation.jl:142; the local cubic
// Hermite with Catmull-Rom slopes of grid_general.cuh), from the interleaved
// float table (E xyz0, B xyz0 per node, 32 bytes).  A particle's stencil is
// 4 x 4 x 4 nodes; a row of 4 nodes along x is 128 contiguous bytes.  Instead
// of each lane gathering its own 64 nodes (64 scattered lines per lane), the
// warp gathers the stencils of its particles four at a time: for each, lane
// l loads nodes (l & 3, (l >> 2) & 3, l >> 4) and (.., .., (l >> 4) + 2) -- 8
// rows of 128 bytes per load instruction -- and weights them; one
// reduce-scatter over the warp sums the four particles' E and B (reduce4x6)
// and the owning lanes fetch theirs.  All 32 lanes of the warp must call it
// together; lanes with want = false only help.
// The weight of node d (0..3) of the 4-node stencil at fraction t of the
// middle cell, w_d(t) = h-basis combination of the Catmull-Rom Hermite cubic
// (grid_general.cuh), as the polynomial c0 + c1 t + c2 t^2 + c3 t^3:
//   w0 = -t/2 + t^2 - t^3/2        w1 = 1 - 5t^2/2 + 3t^3/2
//   w2 =  t/2 + 2t^2 - 3t^3/2      w3 = -t^2/2 + t^3/2
// A lane always takes the same node of every stencil, so its coefficients
// are fixed for the whole kernel and a weight costs three FMAs.
struct CubicW {
    float c0, c1, c2, c3;
};
__device__ __forceinline__ CubicW cubic_coef(int d) {
    return d == 0 ? CubicW{0.0f, -0.5f, 1.0f, -0.5f}
                  : (d == 1 ? CubicW{1.0f, 0.0f, -2.5f, 1.5f}
                            : (d == 2 ? CubicW{0.0f, 0.5f, 2.0f, -1.5f} : CubicW{0.0f, 0.0f, -0.5f, 0.5f}));
}
__device__ __forceinline__ float cubic_w(const CubicW& c, float t) {
    return fmaf(fmaf(fmaf(c.c3, t, c.c2), t, c.c1), t, c.c0);
}

// cell index in [0, n) and fraction in [0, 1) on a periodic axis, from the
// compensated coordinate (positions are wrapped into the box)
__device__ __forceinline__ void cubic_cell(const DevField& g, int a, float hi, float lo, int& i, float& f) {
    AxF o;
    axis32(g, a, hi, lo, o);  // periodic: always in range
    i = o.i0;
    f = o.f;
}

// this lane's weighted share of the stencil of the particle at cell (qi, qj,
// qk), fractions (fx, fy, fz): E in s[0..2], B in s[3..5]
__device__ __forceinline__ void cubic_share(const DevField& g, const float4* tab, int qi, int qj, int qk, float fx,
                                            float fy, float fz, float s[6]) {
    const int lane = threadIdx.x & 31;
    const int dx = lane & 3, dy = (lane >> 2) & 3, dz = lane >> 4;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const float wxy = cubic_w(cubic_coef(dx), fx) * cubic_w(cubic_coef(dy), fy);
    const float w0 = wxy * cubic_w(cubic_coef(dz), fz), w1 = wxy * cubic_w(cubic_coef(dz + 2), fz);
    int ix = qi - 1 + dx, iy = qj - 1 + dy, iz0 = qk - 1 + dz, iz1 = qk + 1 + dz;
    ix += ix < 0 ? nx : 0;
    ix -= ix >= nx ? nx : 0;
    iy += iy < 0 ? ny : 0;
    iy -= iy >= ny ? ny : 0;
    iz0 += iz0 < 0 ? nz : 0;
    iz1 -= iz1 >= nz ? nz : 0;
    const int64_t row = (int64_t)ix + (int64_t)nx * iy;
    const int64_t nxy = (int64_t)nx * ny;
    float4 e0, b0, e1, b1;
    ldg_node8(tab + 2 * (row + nxy * iz0), e0, b0);
    ldg_node8(tab + 2 * (row + nxy * iz1), e1, b1);
    s[0] = fmaf(w0, e0.x, w1 * e1.x);
    s[1] = fmaf(w0, e0.y, w1 * e1.y);
    s[2] = fmaf(w0, e0.z, w1 * e1.z);
    s[3] = fmaf(w0, b0.x, w1 * b1.x);
    s[4] = fmaf(w0, b0.y, w1 * b1.y);
    s[5] = fmaf(w0, b0.z, w1 * b1.z);
}

// Sum s[k][c] (particle k = 0..3, component c = 0..5: E xyz, B xyz) over the
// 32 lanes of the warp by halving (a reduce-scatter): after the exchanges with
// lanes 16, 8 and 4 apart each lane holds three components of one particle
// summed over 8 lanes -- particle 2 b4 + b3, components 3 b2 .. 3 b2 + 2 for
// lane bits b4 b3 b2 -- and two butterfly levels complete the sums: 27
// shuffles for four particles instead of 120.  Returns the three sums.
__device__ __forceinline__ void reduce4x6(const float s[4][6], float out[3]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool b4 = (lane >> 4) & 1, b3 = (lane >> 3) & 1, b2 = (lane >> 2) & 1;
    // lanes 16 apart: keep particles {0, 1} (b4 = 0) or {2, 3}
    float t[2][6];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float keep = b4 ? s[2 + k][c] : s[k][c];
            const float send = b4 ? s[k][c] : s[2 + k][c];
            t[k][c] = keep + __shfl_xor_sync(full, send, 16);
        }
    // lanes 8 apart: keep particle b3 of the pair
    float u[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const float keep = b3 ? t[1][c] : t[0][c];
        const float send = b3 ? t[0][c] : t[1][c];
        u[c] = keep + __shfl_xor_sync(full, send, 8);
    }
    // lanes 4 apart: keep E (b2 = 0) or B
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float keep = b2 ? u[3 + c] : u[c];
        const float send = b2 ? u[c] : u[3 + c];
        out[c] = keep + __shfl_xor_sync(full, send, 4);
    }
#pragma unroll
    for (int o = 2; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c] += __shfl_xor_sync(full, out[c], o);
}

__device__ __forceinline__ void coop_cubic_eval(const DevField& g, const float4* tab, bool want, const CPos& p,
                                                F3& E, F3& B) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int ci[3] = {0, 0, 0};
    float cf[3] = {0.0f, 0.0f, 0.0f};
    if (want) {
        cubic_cell(g, 0, p.hi[0], p.lo[0], ci[0], cf[0]);
        cubic_cell(g, 1, p.hi[1], p.lo[1], ci[1], cf[1]);
        cubic_cell(g, 2, p.hi[2], p.lo[2], ci[2], cf[2]);
    }
    unsigned mask = __ballot_sync(full, want);
    // four particles per round (the last round repeats its final particle)
    while (mask) {
        int q[4];
        q[0] = __ffs(mask) - 1;
        mask &= mask - 1;
#pragma unroll
        for (int k = 1; k < 4; ++k) {
            q[k] = mask ? __ffs(mask) - 1 : q[k - 1];
            mask &= mask - 1;
        }
        float sk[4][6];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            cubic_share(g, tab, __shfl_sync(full, ci[0], q[k]), __shfl_sync(full, ci[1], q[k]),
                        __shfl_sync(full, ci[2], q[k]), __shfl_sync(full, cf[0], q[k]),
                        __shfl_sync(full, cf[1], q[k]), __shfl_sync(full, cf[2], q[k]), sk[k]);
        float r[3];
        reduce4x6(sk, r);
        // the owner of particle k takes E from lane (k >> 1) << 4 | (k & 1) << 3
        // and B from that lane + 4
        int mine = -1;
#pragma unroll
        for (int k = 3; k >= 0; --k)
            if (lane == q[k]) mine = k;
        const int src = mine < 0 ? 0 : (((mine >> 1) << 4) | ((mine & 1) << 3));
        const float ex = __shfl_sync(full, r[0], src), ey = __shfl_sync(full, r[1], src),
                    ez = __shfl_sync(full, r[2], src);
        const float bx = __shfl_sync(full, r[0], src + 4), by = __shfl_sync(full, r[1], src + 4),
                    bz = __shfl_sync(full, r[2], src + 4);
        if (mine >= 0) {
            E = {ex, ey, ez};
            B = {bx, by, bz};
        }
    }
}

// Fixed-step Boris / Multistep in the cubic field, FP32C (compensated float
// positions and velocities, float delta-form rotation), one particle per
// lane, static schedule.  Every lane runs the loop until all lanes of its
// warp are done, so that the cooperative gathers see the whole warp; a lane
// whose particle is done (or that has none) only helps.  The fields are
// static, so the save of r_{k-1} reuses the step's evaluation at r_{k-1}.
// slot k of particle i: state, then the given E and B when save_fields
__device__ __forceinline__ void save_row32(const BorisArgs& a, int W, int64_t i, int64_t k, const CPos& p,
                                           const CV& v, double t, const F3& E, const F3& B) {
    if (k >= a.nslots) {
        set_status(a.status, TP_E_OVERFLOW);
        return;
    }
    const int64_t n = a.n;
    a.t_out[k * n + i] = t;
    double* u = a.u_out + (k * W) * n + i;
    u[0 * n] = cpos_value(a, p, 0);
    u[1 * n] = cpos_value(a, p, 1);
    u[2 * n] = cpos_value(a, p, 2);
    u[3 * n] = (double)v.h.x + (double)v.l.x;
    u[4 * n] = (double)v.h.y + (double)v.l.y;
    u[5 * n] = (double)v.h.z + (double)v.l.z;
    if (a.save_fields) {
        u[6 * n] = E.x;
        u[7 * n] = E.y;
        u[8 * n] = E.z;
        u[9 * n] = B.x;
        u[10 * n] = B.y;
        u[11 * n] = B.z;
    }
}

template <bool MULTI>
__global__ void __launch_bounds__(128, 5) k_cubic32c(BorisArgs a) {
    const int W = 6 + (a.save_fields ? 6 : 0) + (a.save_work ? 4 : 0);
    const uint64_t t_start = globaltimer_ns();
    const int64_t i = take_particle(a, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
    const DevField& g = a.f.B;
    const float4* tab = a.f.ebc32;

    bool active = i < a.n;
    CPos p;
    CV v{};
    for (int c = 0; c < 3; ++c) {
        p.hi[c] = p.lo[c] = 0.0f;
        p.w[c] = 0;
    }
    double dt = 0, t = 0, t1 = 0, t_last = 0;
    float dth = 0, dtl = 0, hstep = 0;
    int64_t it = 1, nt = 0;
    int32_t nout = 0, iout = 0, csave = 0;
    if (active) {
        dt = a.dt_i ? a.dt_i[i] : a.dt;
        t1 = a.tend_i ? a.tend_i[i] : a.t1;
        nt = (fabs(dt) < 10.0 * 2.220446049250313e-16) ? -1 : jl_round((t1 - a.t0) / dt);
        if (nt < 0 && fabs(dt) >= 10.0 * 2.220446049250313e-16) nt = -nt;
        if (nt < 0 || nt > a.maxiters) {
            set_status(a.status, TP_E_ARG);
            a.nsaved[i] = 0;
            a.retcode[i] = TP_RET_DEFAULT;
            a.nsteps[i] = 0;
            particle_done(a, i);
            active = false;
        }
    }
    if (active) {
        dth = (float)dt;
        dtl = (float)(dt - (double)dth);
        hstep = vfac<MULTI>(a, dt);
        nout = (int32_t)calc_nout(nt, a.ssi, a.save_start, a.save_end, a.save_everystep);
        const double* u0 = a.u0 + 6 * i;
        cpos_init(a, p, u0);
        v = cv_from(u0 + 3);
    }
    // v_{-1/2} (and the save of u0 with its fields)
    F3 E{0.0f, 0.0f, 0.0f}, B{0.0f, 0.0f, 0.0f};
    coop_cubic_eval(g, tab, active, p, E, B);
    if (active) {
        if (a.save_start) {
            a.t_out[i] = a.t0;
            if (a.nslots > 0) {
                double* u = a.u_out + i;
                const double* u0 = a.u0 + 6 * i;
                for (int c = 0; c < 6; ++c) u[c * a.n] = u0[c];
                if (a.save_fields) {
                    u[6 * a.n] = E.x; u[7 * a.n] = E.y; u[8 * a.n] = E.z;
                    u[9 * a.n] = B.x; u[10 * a.n] = B.y; u[11 * a.n] = B.z;
                }
            } else {
                set_status(a.status, TP_E_OVERFLOW);
            }
            t_last = a.t0;
            iout = 1;
        }
        v = vel32<MULTI>(v, E, B, a, -0.5 * dt);
        t = a.t0 - 0.5 * dt;
    }
    bool stepping = active && it <= nt;
    bool finishing = active && !stepping;
    for (;;) {
        // ---- one step of _boris_loop! (boris.jl:452-476) for the stepping lanes
        coop_cubic_eval(g, tab, stepping, p, E, B);
        if (stepping) {
            t += dt;
            CV vn = vel32h<MULTI>(v, E, B, a, hstep);
            CPos pn = p;
            cpos_push_cv(a, pn, vn, dth, dtl);
            if (a.term.flags && outside32<FK_GENGRID>(a, pn, vn, t + 0.5 * dt)) {
                finishing = true;
            } else {
                if (a.save_everystep && it > 1 && csave == 0) {
                    iout += 1;
                    if (iout <= nout) {
                        const double t_cur = t - 0.5 * dt;
                        CV vs = vel32<MULTI>(v, E, B, a, 0.5 * dt);
                        save_row32(a, W, i, iout - 1, p, vs, t_cur, E, B);
                        t_last = t_cur;
                    }
                }
                p = pn;
                v = vn;
                it += 1;
                csave += 1;
                if (csave == a.ssi) csave = 0;
                if (it > nt) finishing = true;
                if ((it & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                    set_status(a.status, TP_E_TIMEOUT);
                    finishing = true;
                }
            }
            if (finishing) stepping = false;
        }
        // ---- final save and retcode (boris.jl:522-551) for the lanes that finished
        int64_t final_step = it - 1;
        bool save_final = false;
        double t_final = 0.0;
        if (finishing) {
            save_final = a.save_end || (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
            t_final = (final_step == nt) ? t1 : fma((double)final_step, dt, a.t0);
            save_final = save_final && iout < nout && (iout == 0 || t_last < t_final);
        }
        coop_cubic_eval(g, tab, save_final, p, E, B);
        if (finishing) {
            if (save_final) {
                const double dt_final = t_final - fma((double)final_step - 0.5, dt, a.t0);
                CV vf = vel32<MULTI>(v, E, B, a, dt_final);
                save_row32(a, W, i, iout, p, vf, t_final, E, B);
                iout += 1;
            }
            a.nsaved[i] = (int32_t)iout;
            a.retcode[i] = (int8_t)((iout < nout) ? TP_RET_TERMINATED : TP_RET_SUCCESS);
            a.nsteps[i] = final_step;
            particle_done(a, i);
            finishing = false;
        }
        if (!__any_sync(0xffffffffu, stepping)) break;
    }
}

// ---------------------------------------------------------------- adaptive
template <bool MULTI, bool QUEUE, int FK>
__global__ void __launch_bounds__(TPB_ADAPTIVE32_BOUND(FK), 1) k_adaptive32c(BorisArgs a) {
    using P = Vel32<FK>;
    using V = typename P::V;
    using Fv = typename P::Fv;
    const Saver32<FK> S(a);
    const bool stat = fields_static32(a.f);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double twopi = 6.283185307179586;

    int64_t i = -1;
    CPos p;
    V v{};
    Fv E{0, 0, 0}, B{0, 0, 0};
    double t = 0, t1 = 0, dt = 0, C = 0, ttotal = 0, t_last = 0;
    int64_t it = 0, iout = 0, steps = 0;
    bool ssf = false;
    int ret = TP_RET_SUCCESS;

    for (;;) {
        if (i < 0) {
            i = next_particle32<QUEUE>(a, first);
            if (i >= a.n) break;
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            double dtt = t1 - a.t0;
            double sgn = dtt > 0 ? 1.0 : (dtt < 0 ? -1.0 : 0.0);
            C = (twopi * a.safety * sgn) / fabs(a.q2m);
            const double* u0 = a.u0 + 6 * i;
            cpos_init(a, p, u0);
            v = P::init(u0 + 3);
            t = a.t0;
            ttotal = dtt;
            iout = 0;
            P::fields(a.f, p, t, E, B);
            if (a.save_start) {
                if (a.nslots > 0) {
                    a.t_out[i] = t;
                    double* u = a.u_out + i;
                    for (int c = 0; c < 6; ++c) u[c * a.n] = u0[c];
                    if (a.save_fields) {
                        u[6 * a.n] = E.x; u[7 * a.n] = E.y; u[8 * a.n] = E.z;
                        u[9 * a.n] = B.x; u[10 * a.n] = B.y; u[11 * a.n] = B.z;
                    }
                } else {
                    set_status(a.status, TP_E_OVERFLOW);
                }
                t_last = t;
                iout = 1;
            }
            dt = C / sqrt(P::bmag2(B));
            v = P::template step<MULTI>(v, E, B, a, -0.5 * dt);
            it = 1;
            steps = 0;
            ssf = a.save_end;
            ret = TP_RET_SUCCESS;
        }

        bool done = !(fabs(t - a.t0) < fabs(ttotal));
        if (!done && a.step_cap > 0 && steps >= a.step_cap) {
            ret = TP_RET_MAXITERS;
            done = true;
        }
        if (!done) {
            if (!stat) P::fields(a.f, p, t, E, B);
            if (fabs(t + dt - a.t0) > fabs(ttotal)) {
                double dt_step = t1 - t;
                v = P::template step<MULTI>(v, E, B, a, 0.5 * dt);
                v = P::template step<MULTI>(v, E, B, a, -0.5 * dt_step);
                dt = dt_step;
            }
            if (a.save_everystep && (it - 1) > 0 && (it - 1) % a.ssi == 0) {
                V vs = P::template step<MULTI>(v, E, B, a, 0.5 * dt);
                S.save(i, iout, p, vs, t);
                t_last = t;
                iout += 1;
            }
            Fv Em = E, Bm = B;
            if (!stat) P::fields(a.f, p, t + 0.5 * dt, Em, Bm);
            V v_new = P::template step<MULTI>(v, Em, Bm, a, dt);
            CPos pn = p;
            float dh = (float)dt;
            P::push(a, pn, v_new, dh, (float)(dt - (double)dh), dt);
            double t_next = t + dt;
            if (a.term.flags && outside32<FK>(a, pn, v_new, t_next)) {
                ssf = true;
                ret = TP_RET_TERMINATED;
                done = true;
            } else {
                p = pn;
                t = t_next;
                v = v_new;
                steps += 1;
                P::fields(a.f, p, t, E, B);
                double dt_new = C / sqrt(P::bmag2(B));
                v = P::template step<MULTI>(v, E, B, a, 0.5 * dt);
                v = P::template step<MULTI>(v, E, B, a, -0.5 * dt_new);
                dt = dt_new;
                it += 1;
                if (a.save_everystep && (it - 1) % a.ssi == 0) ssf = true;
                if ((steps & 1023) == 0 && globaltimer_ns() - t_start > a.budget_ns) {
                    set_status(a.status, TP_E_TIMEOUT);
                    ret = TP_RET_DEFAULT;
                    done = true;
                }
            }
        }
        if (done) {
            if (ssf && (iout == 0 || t_last != t)) {
                if (!stat) P::fields(a.f, p, t, E, B);
                V vf = P::template step<MULTI>(v, E, B, a, 0.5 * dt);
                S.save(i, iout, p, vf, t);
                iout += 1;
            }
            a.nsaved[i] = (int32_t)iout;
            a.retcode[i] = (int8_t)ret;
            a.nsteps[i] = steps;
            particle_done(a, i);
            i = -1;
        }
    }
}

// ---------------------------------------------------------------- launchers
// Two particles per thread are compiled for the analytic-field fixed-step
// kernels (no field memory: a slot without a particle computes without
// touching memory); everything else runs one particle per thread.
template <bool MULTI, bool QUEUE, int FK>
static const void* kernel_ptr32(bool adaptive, int ppt) {
    if (adaptive) return (const void*)k_adaptive32c<MULTI, QUEUE, FK>;
    if (FK == FK_ANALYTIC && ppt == 2) return (const void*)k_fixed32c_slots<MULTI, QUEUE, FK, 2>;
    return (const void*)k_fixed32c<MULTI, QUEUE, FK>;
}

template <bool MULTI, bool QUEUE>
static const void* pick_fk32(bool adaptive, int fk, int ppt) {
    if (fk == FK_ANALYTIC) return kernel_ptr32<MULTI, QUEUE, FK_ANALYTIC>(adaptive, ppt);
    if (fk == FK_EBGRID) return kernel_ptr32<MULTI, QUEUE, FK_EBGRID>(adaptive, 1);
    if (fk == FK_GENGRID) return kernel_ptr32<MULTI, QUEUE, FK_GENGRID>(adaptive, 1);
    return kernel_ptr32<MULTI, QUEUE, FK_GENERIC>(adaptive, 1);
}

// fixed steps in static cubic grids with the interleaved table
static bool cubic_coop_kernel(const BorisArgs& a) {
    return a.f.ebc32 != nullptr && (a.alg == TP_ALG_BORIS || a.alg == TP_ALG_MULTISTEP);
}

bool fp32c_cubic_coop(const BorisArgs& a) { return cubic_coop_kernel(a); }

static const void* select_kernel32(const BorisArgs& a, bool queue) {
    const bool multi = a.alg == TP_ALG_MULTISTEP || a.alg == TP_ALG_ADAPTIVE_MULTISTEP;
    const bool adaptive = a.alg == TP_ALG_ADAPTIVE || a.alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (cubic_coop_kernel(a)) return multi ? (const void*)k_cubic32c<true> : (const void*)k_cubic32c<false>;
    const int fk = field_config_of(a.f);
    const int ppt = a.ppt;
    if (multi) return queue ? pick_fk32<true, true>(adaptive, fk, ppt) : pick_fk32<true, false>(adaptive, fk, ppt);
    return queue ? pick_fk32<false, true>(adaptive, fk, ppt) : pick_fk32<false, false>(adaptive, fk, ppt);
}

cudaError_t launch_boris_fp32c(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s) {
    const void* k = select_kernel32(a, a.use_queue != 0);
    void* args[] = {const_cast<BorisArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(c.grid), dim3(c.block), args, 0, s);
}

cudaError_t prime_boris_fp32c(const BorisArgs& a) {
    cudaFuncAttributes at;
    return cudaFuncGetAttributes(&at, select_kernel32(a, a.use_queue != 0));
}

int occupancy_boris_fp32c(const BorisArgs& a, int block) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, select_kernel32(a, true), block, 0);
    return nb;
}

}  // namespace tpb
