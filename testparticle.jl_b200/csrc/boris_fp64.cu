// boris_fp64.cu -- float64 full-orbit push kernels (the drop-in path).
//
// Compiled with -fmad=false: the arithmetic follows the reference's operation
// order (see fields64.cuh).  One thread owns one particle at a time and keeps
// its whole state in registers for all steps; saves go straight from the
// kernel into slot-major output arrays (coalesced across the warp), replacing
// the reference GPU path's one launch + host copy per step
// (src/boris/boris_kernel.jl:170-198).
//
// Schedules.  STATIC: thread g owns particle g.  QUEUE: a persistent grid of
// threads pulls particle indices from a device counter; a lane whose particle
// finishes (end of tspan, isoutside, step cap) fetches the next one in the
// same loop iteration, so lanes stay busy when lifetimes are uneven.
//
// Kernels (MULTI: Multistep update; QUEUE: schedule; FK: field configuration,
// see tp_device.cuh):
//   k_fixed64<MULTI, QUEUE, FK, PPT>  _boris_single + _boris_loop!  (boris.jl:445-557)
//                                  with Boris (boris.jl:19-45) or
//                                  Multistep (multistep_boris.jl:65-142) updates
//   k_adaptive64<MULTI, QUEUE, FK> _adaptive_boris_single (adaptive_boris.jl:145-266)
#include "fields64.cuh"
#include "tp_launch.h"

namespace tpb {

namespace {

template <int FK>
struct Saver64 {
    const BorisArgs& a;
    int W;
    __device__ Saver64(const BorisArgs& a_)
        : a(a_), W(6 + (a_.save_fields ? 6 : 0) + (a_.save_work ? 4 : 0)) {}
    // slot k of particle i: state, then E and B at (r, t) when save_fields
    // (_prepare_saved_data, boris.jl:405-440); the four work-rate columns of
    // save_work are filled by a post-pass over the saved states
    __device__ __forceinline__ void save(int64_t i, int64_t k, D3 r, D3 v, double t) const {
        if (k >= a.nslots) {
            set_status(a.status, TP_E_OVERFLOW);
            return;
        }
        const int64_t n = a.n;
        a.t_out[k * n + i] = t;
        double* u = a.u_out + (k * W) * n + i;
        u[0 * n] = r.x;
        u[1 * n] = r.y;
        u[2 * n] = r.z;
        u[3 * n] = v.x;
        u[4 * n] = v.y;
        u[5 * n] = v.z;
        if (a.save_fields) {
            D3 E, B;
            eval_EB64t<FK>(a.f, r, t, E, B);
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
__device__ __forceinline__ int64_t next_particle(const BorisArgs& a, int64_t& first) {
    if (!QUEUE) {
        int64_t g = first;
        first = a.n;  // static: one particle per thread
        return take_particle(a, g);
    }
    return take_particle(a, (int64_t)atomicAdd(a.queue, 1ULL));
}

}  // namespace

// ---------------------------------------------------------------- fixed step
template <bool MULTI, bool QUEUE, int FK>
__global__ void __launch_bounds__(TPB_FIXED_BOUND(FK), 1) k_fixed64(BorisArgs a) {
    const Saver64<FK> S(a);
    const bool stat = fields_static(a.f);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;

    // per-particle state
    int64_t i = -1;
    D3 r{0, 0, 0}, v{0, 0, 0};
    double dt = 0, t = 0, t1 = 0, t_last = 0;
    int64_t it = 0, nt = 0;
    int32_t nout = 0, iout = 0, csave = 0;

    for (;;) {
        if (i < 0) {
            i = next_particle<QUEUE>(a, first);
            if (i >= a.n) break;
            // ---- setup: _boris_single (boris.jl:480-514)
            dt = a.dt_i ? a.dt_i[i] : a.dt;
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            if (fabs(dt) < 10.0 * 2.220446049250313e-16) {
                set_status(a.status, TP_E_ARG);
                a.nsaved[i] = 0;
                a.retcode[i] = TP_RET_DEFAULT;
                a.nsteps[i] = 0;
                particle_done(a, i);
                i = -1;
                continue;
            }
            nt = jl_round((t1 - a.t0) / dt);
            if (nt < 0) nt = -nt;
            if (nt > a.maxiters) {
                set_status(a.status, TP_E_ARG);
                a.nsaved[i] = 0;
                a.retcode[i] = TP_RET_DEFAULT;
                a.nsteps[i] = 0;
                particle_done(a, i);
                i = -1;
                continue;
            }
            nout = (int32_t)calc_nout(nt, a.ssi, a.save_start, a.save_end, a.save_everystep);
            const double* u0 = a.u0 + 6 * i;
            r = {u0[0], u0[1], u0[2]};
            v = {u0[3], u0[4], u0[5]};
            iout = 0;
            if (a.save_start) {
                S.save(i, 0, r, v, a.t0);
                t_last = a.t0;
                iout = 1;
            }
            D3 E, B;
            eval_EB64t<FK>(a.f, r, a.t0, E, B);
            v = vel_update64<MULTI>(v, E, B, a.q2m, -0.5 * dt, a.order, a.nsub);
            it = 1;
            t = a.t0 - 0.5 * dt;
            csave = 0;  // (it - 1) % ssi
        }

        bool done = it > nt;
        if (!done) {
            // ---- one step of _boris_loop! (boris.jl:452-476); v stays the
            // pre-step velocity (the reference's v_prev) until the step is
            // accepted, which serves both the save and the termination rollback
            t += dt;
            D3 E, B;
            eval_EB64t<FK>(a.f, r, t, E, B);
            D3 vn = vel_update64<MULTI>(v, E, B, a.q2m, dt, a.order, a.nsub);
            D3 r_next = r + vn * dt;
            double t_next = t + 0.5 * dt;
            if (a.term.flags && outside64(a.term, r_next, vn, t_next)) {
                done = true;
            } else {
                if (a.save_everystep && it > 1 && csave == 0) {
                    iout += 1;
                    if (iout <= nout) {
                        double t_cur = t - 0.5 * dt;
                        if (!stat) eval_EB64t<FK>(a.f, r, t_cur, E, B);
                        D3 v_save = vel_update64<MULTI>(v, E, B, a.q2m, 0.5 * dt, a.order, a.nsub);
                        S.save(i, iout - 1, r, v_save, t_cur);
                        t_last = t_cur;
                    }
                }
                r = r_next;
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
            // ---- final save and retcode (boris.jl:522-551)
            int64_t final_step = it - 1;
            bool save_final = a.save_end ||
                              (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
            if (iout < nout && save_final) {
                double t_final = (final_step == nt) ? t1 : fma((double)final_step, dt, a.t0);
                if (iout == 0 || t_last < t_final) {
                    double dt_final = t_final - fma((double)final_step - 0.5, dt, a.t0);
                    D3 E, B;
                    eval_EB64t<FK>(a.f, r, t_final, E, B);
                    D3 vf = vel_update64<MULTI>(v, E, B, a.q2m, dt_final, a.order, a.nsub);
                    S.save(i, iout, r, vf, t_final);
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
// PPT particles per thread ("slots") in lock step, as in boris_fp32c.cu: each
// iteration refills idle slots, computes every slot's step as one
// straight-line block (independent float64 chains the scheduler can
// interleave), then commits each slot.  The arithmetic of a slot is that of
// one particle per thread, so the results do not depend on PPT.  Static
// schedule: slot k of global thread g owns particle g + k * (threads in the grid).
template <bool MULTI, bool QUEUE, int FK, int PPT>
__global__ void __launch_bounds__(TPB_MAXT(FK) / PPT, 1) k_fixed64_slots(BorisArgs a) {
    const Saver64<FK> S(a);
    const uint64_t t_start = globaltimer_ns();
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;

    // per-slot particle state
    int64_t first[PPT], i[PPT];
    D3 r[PPT], v[PPT];
    double dt[PPT], t[PPT], t1[PPT], t_last[PPT];
    int64_t it[PPT], nt[PPT];
    int32_t nout[PPT], iout[PPT], csave[PPT];
    bool dead[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        first[k] = g + k * gstride;
        i[k] = -1;
        dead[k] = false;
        r[k] = v[k] = D3{0.0, 0.0, 0.0};
        dt[k] = t[k] = t1[k] = t_last[k] = 0.0;
        it[k] = nt[k] = 0;
        nout[k] = iout[k] = csave[k] = 0;
    }

    for (;;) {
        // ---- refill idle slots: _boris_single (boris.jl:480-514)
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            while (!dead[k] && i[k] < 0) {
                i[k] = next_particle<QUEUE>(a, first[k]);
                if (i[k] >= a.n) {
                    dead[k] = true;
                    break;
                }
                const int64_t ii = i[k];
                dt[k] = a.dt_i ? a.dt_i[ii] : a.dt;
                t1[k] = a.tend_i ? a.tend_i[ii] : a.t1;
                if (fabs(dt[k]) < 10.0 * 2.220446049250313e-16) {
                    set_status(a.status, TP_E_ARG);
                    a.nsaved[ii] = 0;
                    a.retcode[ii] = TP_RET_DEFAULT;
                    a.nsteps[ii] = 0;
                    particle_done(a, ii);
                    i[k] = -1;
                    continue;
                }
                nt[k] = jl_round((t1[k] - a.t0) / dt[k]);
                if (nt[k] < 0) nt[k] = -nt[k];
                if (nt[k] > a.maxiters) {
                    set_status(a.status, TP_E_ARG);
                    a.nsaved[ii] = 0;
                    a.retcode[ii] = TP_RET_DEFAULT;
                    a.nsteps[ii] = 0;
                    particle_done(a, ii);
                    i[k] = -1;
                    continue;
                }
                nout[k] = (int32_t)calc_nout(nt[k], a.ssi, a.save_start, a.save_end, a.save_everystep);
                const double* u0 = a.u0 + 6 * ii;
                r[k] = {u0[0], u0[1], u0[2]};
                v[k] = {u0[3], u0[4], u0[5]};
                iout[k] = 0;
                if (a.save_start) {
                    S.save(ii, 0, r[k], v[k], a.t0);
                    t_last[k] = a.t0;
                    iout[k] = 1;
                }
                D3 E, B;
                eval_EB64t<FK>(a.f, r[k], a.t0, E, B);
                v[k] = vel_update64<MULTI>(v[k], E, B, a.q2m, -0.5 * dt[k], a.order, a.nsub);
                it[k] = 1;
                t[k] = a.t0 - 0.5 * dt[k];
                csave[k] = 0;  // (it - 1) % ssi
            }
        }
        bool any = false;
#pragma unroll
        for (int k = 0; k < PPT; ++k) any = any || !dead[k];
        if (!any) break;

        // ---- one step of _boris_loop! (boris.jl:452-476) for every slot; v
        // stays the pre-step velocity (the reference's v_prev) until the step
        // is accepted, which serves both the save and the termination rollback
        D3 vn[PPT], r_next[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            D3 E, B;
            eval_EB64t<FK>(a.f, r[k], t[k] + dt[k], E, B);
            vn[k] = vel_update64<MULTI>(v[k], E, B, a.q2m, dt[k], a.order, a.nsub);
            r_next[k] = r[k] + vn[k] * dt[k];
        }

#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            if (dead[k]) continue;
            const int64_t ii = i[k];
            bool done = it[k] > nt[k];
            if (!done) {
                t[k] += dt[k];
                const double t_next = t[k] + 0.5 * dt[k];
                if (a.term.flags && outside64(a.term, r_next[k], vn[k], t_next)) {
                    done = true;
                } else {
                    if (a.save_everystep && it[k] > 1 && csave[k] == 0) {
                        iout[k] += 1;
                        if (iout[k] <= nout[k]) {
                            const double t_cur = t[k] - 0.5 * dt[k];
                            D3 E, B;
                            eval_EB64t<FK>(a.f, r[k], t_cur, E, B);
                            D3 v_save = vel_update64<MULTI>(v[k], E, B, a.q2m, 0.5 * dt[k], a.order, a.nsub);
                            S.save(ii, iout[k] - 1, r[k], v_save, t_cur);
                            t_last[k] = t_cur;
                        }
                    }
                    r[k] = r_next[k];
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
                // ---- final save and retcode (boris.jl:522-551)
                const int64_t final_step = it[k] - 1;
                const bool save_final = a.save_end ||
                                        (a.save_everystep && final_step > 0 && final_step % a.ssi == 0);
                if (iout[k] < nout[k] && save_final) {
                    const double t_final = (final_step == nt[k]) ? t1[k] : fma((double)final_step, dt[k], a.t0);
                    if (iout[k] == 0 || t_last[k] < t_final) {
                        const double dt_final = t_final - fma((double)final_step - 0.5, dt[k], a.t0);
                        D3 E, B;
                        eval_EB64t<FK>(a.f, r[k], t_final, E, B);
                        D3 vf = vel_update64<MULTI>(v[k], E, B, a.q2m, dt_final, a.order, a.nsub);
                        S.save(ii, iout[k], r[k], vf, t_final);
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

// ---------------------------------------------------------------- adaptive
template <bool MULTI, bool QUEUE, int FK>
__global__ void __launch_bounds__(TPB_ADAPTIVE64_BOUND(FK), 1) k_adaptive64(BorisArgs a) {
    const Saver64<FK> S(a);
    const bool stat = fields_static(a.f);
    const uint64_t t_start = globaltimer_ns();
    int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double twopi = 6.283185307179586;

    int64_t i = -1;
    D3 r{0, 0, 0}, v{0, 0, 0};
    D3 E{0, 0, 0}, B{0, 0, 0};  // fields at (r, t) when static
    double t = 0, t1 = 0, dt = 0, C = 0, ttotal = 0, t_last = 0;
    int64_t it = 0, iout = 0, steps = 0;
    bool ssf = false;
    int ret = TP_RET_SUCCESS;

    for (;;) {
        if (i < 0) {
            i = next_particle<QUEUE>(a, first);
            if (i >= a.n) break;
            // ---- setup (adaptive_boris.jl:149-196)
            t1 = a.tend_i ? a.tend_i[i] : a.t1;
            double dtt = t1 - a.t0;
            double sgn = dtt > 0 ? 1.0 : (dtt < 0 ? -1.0 : 0.0);
            C = (twopi * a.safety * sgn) / fabs(a.q2m);
            const double* u0 = a.u0 + 6 * i;
            r = {u0[0], u0[1], u0[2]};
            v = {u0[3], u0[4], u0[5]};
            t = a.t0;
            ttotal = dtt;
            iout = 0;
            if (a.save_start) {
                S.save(i, 0, r, v, t);
                t_last = t;
                iout = 1;
            }
            eval_EB64t<FK>(a.f, r, t, E, B);
            dt = C / norm(B);
            v = vel_update64<MULTI>(v, E, B, a.q2m, -0.5 * dt, a.order, a.nsub);
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
            // ---- one iteration of the while loop (adaptive_boris.jl:197-248)
            if (!stat) eval_EB64t<FK>(a.f, r, t, E, B);
            if (fabs(t + dt - a.t0) > fabs(ttotal)) {
                double dt_step = t1 - t;
                v = vel_update64<MULTI>(v, E, B, a.q2m, 0.5 * dt, a.order, a.nsub);
                v = vel_update64<MULTI>(v, E, B, a.q2m, -0.5 * dt_step, a.order, a.nsub);
                dt = dt_step;
            }
            if (a.save_everystep && (it - 1) > 0 && (it - 1) % a.ssi == 0) {
                D3 v_save = vel_update64<MULTI>(v, E, B, a.q2m, 0.5 * dt, a.order, a.nsub);
                S.save(i, iout, r, v_save, t);
                t_last = t;
                iout += 1;
            }
            double t_mid = t + 0.5 * dt;
            D3 Em = E, Bm = B;
            if (!stat) eval_EB64t<FK>(a.f, r, t_mid, Em, Bm);
            D3 v_new = vel_update64<MULTI>(v, Em, Bm, a.q2m, dt, a.order, a.nsub);
            D3 r_next = r + v_new * dt;
            double t_next = t + dt;
            if (a.term.flags && outside64(a.term, r_next, v_new, t_next)) {
                ssf = true;
                ret = TP_RET_TERMINATED;
                done = true;
            } else {
                r = r_next;
                t = t_next;
                v = v_new;
                steps += 1;
                eval_EB64t<FK>(a.f, r, t, E, B);
                double dt_new = C / norm(B);
                v = vel_update64<MULTI>(v, E, B, a.q2m, 0.5 * dt, a.order, a.nsub);
                v = vel_update64<MULTI>(v, E, B, a.q2m, -0.5 * dt_new, a.order, a.nsub);
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
            // ---- final save (adaptive_boris.jl:250-259)
            if (ssf && (iout == 0 || t_last != t)) {
                if (!stat) eval_EB64t<FK>(a.f, r, t, E, B);
                D3 vf = vel_update64<MULTI>(v, E, B, a.q2m, 0.5 * dt, a.order, a.nsub);
                S.save(i, iout, r, vf, t);
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
// kernels only (see boris_fp32c.cu).
template <bool MULTI, bool QUEUE, int FK>
static const void* kernel_ptr64(bool adaptive, int ppt) {
    if (adaptive) return (const void*)k_adaptive64<MULTI, QUEUE, FK>;
    if (FK == FK_ANALYTIC && ppt == 2) return (const void*)k_fixed64_slots<MULTI, QUEUE, FK, 2>;
    return (const void*)k_fixed64<MULTI, QUEUE, FK>;
}

template <bool MULTI, bool QUEUE>
static const void* pick_fk64(bool adaptive, int fk, int ppt) {
    if (fk == FK_ANALYTIC) return kernel_ptr64<MULTI, QUEUE, FK_ANALYTIC>(adaptive, ppt);
    if (fk == FK_EBGRID) return kernel_ptr64<MULTI, QUEUE, FK_EBGRID>(adaptive, 1);
    if (fk == FK_GENGRID) return kernel_ptr64<MULTI, QUEUE, FK_GENGRID>(adaptive, 1);
    return kernel_ptr64<MULTI, QUEUE, FK_GENERIC>(adaptive, 1);
}

static const void* select_kernel64(const BorisArgs& a, bool queue) {
    const bool multi = a.alg == TP_ALG_MULTISTEP || a.alg == TP_ALG_ADAPTIVE_MULTISTEP;
    const bool adaptive = a.alg == TP_ALG_ADAPTIVE || a.alg == TP_ALG_ADAPTIVE_MULTISTEP;
    const int fk = field_config_of(a.f);
    const int ppt = a.ppt;
    if (multi) return queue ? pick_fk64<true, true>(adaptive, fk, ppt) : pick_fk64<true, false>(adaptive, fk, ppt);
    return queue ? pick_fk64<false, true>(adaptive, fk, ppt) : pick_fk64<false, false>(adaptive, fk, ppt);
}

cudaError_t launch_boris_fp64(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s) {
    const void* k = select_kernel64(a, a.use_queue != 0);
    void* args[] = {const_cast<BorisArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(c.grid), dim3(c.block), args, 0, s);
}

cudaError_t prime_boris_fp64(const BorisArgs& a) {
    cudaFuncAttributes at;
    return cudaFuncGetAttributes(&at, select_kernel64(a, a.use_queue != 0));
}

int occupancy_boris_fp64(const BorisArgs& a, int block) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, select_kernel64(a, true), block, 0);
    return nb;
}

}  // namespace tpb
