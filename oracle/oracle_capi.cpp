// oracle_capi.cpp -- C entry points of the CPU oracle (liboracle.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py, never by the product.
//
// The entry points take the same descriptors as the CUDA library
// (include/tp_abi.h) and write the same slot-major output layout, so the two
// can be compared element by element.  An OpenMP loop over particles stands
// in for the reference's EnsembleThreads (src/boris/boris.jl:189-215:
// Threads.@threads over index chunks).  Fields and the termination predicate
// may instead be given as C callbacks, which is how the tests restate the
// reference tests' Julia closures.
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "tp_oracle.hpp"

using namespace orc;

extern "C" {

typedef struct orc_field_cb {
    field_cb f;
    jac_cb j;
    void* user;
} orc_field_cb;

typedef struct orc_term_cb {
    outside_cb f;
    void* user;
} orc_term_cb;
}

namespace {

template <class D>
std::unique_ptr<Field> make_general(const tp_field_desc* d) {
    auto* f = new GeneralGridField<D>();
    f->order = d->order;
    f->geom = d->geometry;
    const bool sph = d->geometry == TP_GRID_SPHERICAL || d->geometry == TP_GRID_SPHERICAL_SCALAR;
    f->ndim = sph ? 3 : (d->ndim == 0 ? 3 : d->ndim);
    f->dir = d->dir;
    for (int a = 0; a < 3; ++a) {
        f->n[a] = d->n[a];
        f->abc[a] = d->bc;
        if (d->axis[a]) {
            f->coords[a].assign(d->axis[a], d->axis[a] + d->n[a]);
            f->x0[a] = d->axis[a][0];
            f->inv_dx[a] = 1.0;
        } else {
            f->x0[a] = d->origin[a];
            f->inv_dx[a] = d->n[a] == 1 ? 1.0 : 1.0 / d->spacing[a];
        }
    }
    if (sph) {
        f->abc[0] = TP_BC_FILL_NAN;
        f->abc[1] = TP_BC_FILL_NAN;
        f->abc[2] = TP_BC_PERIODIC_INCLUSIVE;
    }
    f->data = (const D*)d->data;
    return std::unique_ptr<Field>(f);
}

std::unique_ptr<Field> make_field(const tp_field_desc* d, const orc_field_cb* cb) {
    if (cb && cb->f) {
        auto* f = new CallbackField();
        f->f = cb->f;
        f->jf = cb->j;
        f->user = cb->user;
        return std::unique_ptr<Field>(f);
    }
    if (!d || d->kind == TP_FIELD_ZERO) return std::unique_ptr<Field>(new ZeroField());
    switch (d->kind) {
        case TP_FIELD_UNIFORM:
            return std::unique_ptr<Field>(new UniformField({d->value[0], d->value[1], d->value[2]}));
        case TP_FIELD_AFFINE: {
            auto* f = new AffineField();
            f->f0 = {d->value[0], d->value[1], d->value[2]};
            std::memcpy(f->Jm.a, d->jac, sizeof(f->Jm.a));
            f->rate = {d->rate[0], d->rate[1], d->rate[2]};
            return std::unique_ptr<Field>(f);
        }
        case TP_FIELD_SERIES: {
            if (d->nseries < 1 || !d->series || !d->series_times) return nullptr;
            auto* f = new SeriesField();
            for (int64_t k = 0; k < d->nseries; ++k) {
                if (d->series[k].kind == TP_FIELD_SERIES) {
                    delete f;
                    return nullptr;
                }
                f->times.push_back(d->series_times[k]);
                f->snaps.push_back(make_field(&d->series[k], nullptr));
                if (!f->snaps.back()) {
                    delete f;
                    return nullptr;
                }
            }
            return std::unique_ptr<Field>(f);
        }
        case TP_FIELD_QUADRATIC: {
            auto* f = new QuadraticField();
            for (int k = 0; k < 3; ++k) {
                f->v[k] = d->value[k];
                f->rate[k] = d->rate[k];
            }
            std::memcpy(f->J, d->jac, sizeof(f->J));
            std::memcpy(f->Q, d->quad, sizeof(f->Q));
            return std::unique_ptr<Field>(f);
        }
        case TP_FIELD_DIPOLE: {
            auto* f = new DipoleField();
            f->m = {d->moment[0], d->moment[1], d->moment[2]};
            f->c = {d->center[0], d->center[1], d->center[2]};
            f->coef = d->coef;
            return std::unique_ptr<Field>(f);
        }
        case TP_FIELD_GRID: {
            const int ndim = d->ndim == 0 ? 3 : d->ndim;
            const bool general = d->order != TP_ORDER_LINEAR || d->geometry != TP_GRID_CARTESIAN || ndim != 3 ||
                                 d->bc == TP_BC_PERIODIC_INCLUSIVE || d->axis[0] || d->axis[1] || d->axis[2];
            if (general) {
                if (d->dtype == TP_DTYPE_F32) return make_general<float>(d);
                return make_general<double>(d);
            }
            if (d->dtype == TP_DTYPE_F32) {
                auto* f = new GridField<float>();
                for (int a = 0; a < 3; ++a) {
                    f->n[a] = d->n[a];
                    f->x0[a] = d->origin[a];
                    f->inv_dx[a] = 1.0 / d->spacing[a];
                }
                f->bc = d->bc;
                f->data = (const float*)d->data;
                return std::unique_ptr<Field>(f);
            } else {
                auto* f = new GridField<double>();
                for (int a = 0; a < 3; ++a) {
                    f->n[a] = d->n[a];
                    f->x0[a] = d->origin[a];
                    f->inv_dx[a] = 1.0 / d->spacing[a];
                }
                f->bc = d->bc;
                f->data = (const double*)d->data;
                return std::unique_ptr<Field>(f);
            }
        }
    }
    return nullptr;
}

Term make_term(const tp_term_desc* d, const orc_term_cb* cb) {
    Term t;
    std::memset(&t.d, 0, sizeof(t.d));
    if (d) t.d = *d;
    if (cb && cb->f) {
        t.cb = cb->f;
        t.user = cb->user;
    }
    return t;
}

// Copy one trajectory into the slot-major output:
//   t_out[k*n + i], u_out[(k*W + c)*n + i]
bool store(const Traj& tr, int64_t i, int64_t n, int W, int64_t nslots, double* t_out,
           double* u_out, int32_t* nsaved, int8_t* retcode, int64_t* nsteps) {
    int64_t ns = (int64_t)tr.t.size();
    if (nsaved) nsaved[i] = (int32_t)ns;
    if (retcode) retcode[i] = (int8_t)tr.retcode;
    if (nsteps) nsteps[i] = tr.nsteps;
    int64_t m = ns < nslots ? ns : nslots;
    for (int64_t k = 0; k < m; ++k) {
        if (t_out) t_out[k * n + i] = tr.t[k];
        if (u_out)
            for (int c = 0; c < W; ++c) u_out[(k * W + c) * n + i] = tr.u[k * W + c];
    }
    return ns <= nslots;
}

}  // namespace

extern "C" {

int orc_version(void) { return TP_ABI_VERSION; }

int orc_max_threads(void) { return omp_get_max_threads(); }

// nt and nout of _prepare_checks (src/boris/boris.jl:345-403).  Returns
// TP_E_ARG for |dt| < 10 eps or nt > maxiters.
int orc_boris_counts(double t0, double t1, double dt, int64_t maxiters, int64_t ssi,
                     int save_start, int save_end, int save_everystep, int64_t* nt_out,
                     int64_t* nout_out) {
    if (std::fabs(dt) < 10.0 * 2.220446049250313e-16) return TP_E_ARG;
    if (ssi < 1) return TP_E_ARG;
    double ttotal = t1 - t0;
    int64_t nt = jl_round(ttotal / dt);
    if (nt < 0) nt = -nt;
    if (nt > maxiters) return TP_E_ARG;
    *nt_out = nt;
    *nout_out = calculate_nout(nt, ssi, save_start != 0, save_end != 0, save_everystep != 0);
    return TP_OK;
}

}  // extern "C"

namespace {

// ---- forward-mode tangent of the fixed-step Boris map -------------------
// Stands in for ForwardDiff through the reference solver (Julia is absent):
// the primal is the oracle's own Boris update in the reference's order, and
// the tangent follows it operation by operation.

// Field tangent at r along a direction: J(r) rdot plus the direction field
// (node-value and parameter perturbations) at r.
V3d field_tangent(const Field& f, const Field* dgrid, const Field* dpar, V3d r, V3d rdot, double t) {
    V3d F;
    M3 J;
    f.jac(r, t, F, J);
    V3d o{(J(0, 0) * rdot.x + J(0, 1) * rdot.y) + J(0, 2) * rdot.z,
          (J(1, 0) * rdot.x + J(1, 1) * rdot.y) + J(1, 2) * rdot.z,
          (J(2, 0) * rdot.x + J(2, 1) * rdot.y) + J(2, 2) * rdot.z};
    if (dgrid) o = o + dgrid->eval(r, t);
    if (dpar) o = o + dpar->eval(r, t);
    return o;
}

// boris_velocity_update (boris.jl:19-31) and its derivative:
//   t = hB, s = 2t/(1+|t|^2), vm = v + hE, vp = vm + vm x t,
//   v+ = vm + vp x s, v_new = v+ + hE
void boris_update_tangent(V3d v, V3d vd, V3d E, V3d Ed, V3d B, V3d Bd, double h, V3d& vn, V3d& vnd) {
    vn = boris_velocity_update(v, E, B, h);
    V3d t = h * B, td = h * Bd;
    double den = 1.0 + abs2sum(t);
    double dden = 2.0 * dot(t, td);
    V3d s = (2.0 * t) / den;
    V3d sd = (2.0 / den) * td - ((2.0 * dden) / (den * den)) * t;
    V3d vm = v + h * E, vmd = vd + h * Ed;
    V3d vp = vm + cross(vm, t);
    V3d vpd = (vmd + cross(vmd, t)) + cross(vm, td);
    V3d vplusd = (vmd + cross(vpd, s)) + cross(vp, sd);
    vnd = vplusd + h * Ed;
}

// The direction field of a parameter perturbation: the dipole's moment, or
// a uniform offset for every other kind.
std::unique_ptr<Field> param_direction(const tp_field_desc* d, const double* dp) {
    if (!dp || (dp[0] == 0.0 && dp[1] == 0.0 && dp[2] == 0.0)) return nullptr;
    if (d && d->kind == TP_FIELD_DIPOLE) {
        auto* f = new DipoleField();
        f->m = {dp[0], dp[1], dp[2]};
        f->c = {d->center[0], d->center[1], d->center[2]};
        f->coef = d->coef;
        return std::unique_ptr<Field>(f);
    }
    return std::unique_ptr<Field>(new UniformField({dp[0], dp[1], dp[2]}));
}

// The direction field of node-value perturbations of a grid field.
std::unique_ptr<Field> grid_direction(const tp_field_desc* d, const double* nodes) {
    if (!nodes || !d || d->kind != TP_FIELD_GRID) return nullptr;
    tp_field_desc g = *d;
    g.dtype = TP_DTYPE_F64;
    g.data = nodes;
    return make_field(&g, nullptr);
}

}  // namespace

extern "C" {

// Final save (x_N, v_N) of the fixed-step Boris solve of orc_boris_run
// (boris.jl:445-557 with save_end, no termination, static fields) and its
// directional derivative along (du0, dE_nodes, dB_nodes, dparam):
//   du0       N x 6 tangent of the initial states (NULL = 0)
//   dE_nodes, dB_nodes  tangents of a grid field's node values, float64 in
//             the field's data layout (NULL = 0)
//   dparam    6: tangent of (E, B) parameters -- the dipole moment for a
//             dipole, else a uniform offset (NULL = 0)
// uN, duN: N x 6.
int orc_boris_jvp(const tp_run_desc* d, const tp_field_desc* Ed, const tp_field_desc* Bd,
                  const double* u0, const double* du0, const double* dE_nodes, const double* dB_nodes,
                  const double* dparam, int64_t n, int nthreads, double* uN, double* duN) {
    std::unique_ptr<Field> E = make_field(Ed, nullptr), B = make_field(Bd, nullptr);
    if (!E || !B) return TP_E_ARG;
    if (d->alg != TP_ALG_BORIS) return TP_E_UNSUPPORTED;
    int64_t nt, nout;
    int st = orc_boris_counts(d->t0, d->t1, d->dt, d->maxiters, 1, 0, 1, 0, &nt, &nout);
    if (st != TP_OK) return st;
    std::unique_ptr<Field> gE = grid_direction(Ed, dE_nodes), gB = grid_direction(Bd, dB_nodes);
    std::unique_ptr<Field> pE = param_direction(Ed, dparam), pB = param_direction(Bd, dparam ? dparam + 3 : nullptr);
    const double dt = d->dt, t0 = d->t0, h_loop = d->q2m * 0.5 * dt;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int64_t i = 0; i < n; ++i) {
        const double* ui = u0 + 6 * i;
        V3d r{ui[0], ui[1], ui[2]}, v{ui[3], ui[4], ui[5]};
        V3d rd{0, 0, 0}, vd{0, 0, 0};
        if (du0) {
            const double* q = du0 + 6 * i;
            rd = {q[0], q[1], q[2]};
            vd = {q[3], q[4], q[5]};
        }
        auto update = [&](double h, double t) {
            V3d Ev = E->eval(r, t), Bv = B->eval(r, t);
            V3d Et = field_tangent(*E, gE.get(), pE.get(), r, rd, t);
            V3d Bt = field_tangent(*B, gB.get(), pB.get(), r, rd, t);
            V3d vn, vnd;
            boris_update_tangent(v, vd, Ev, Et, Bv, Bt, h, vn, vnd);
            v = vn;
            vd = vnd;
        };
        update(d->q2m * 0.5 * (-0.5 * dt), t0);  // v_{-1/2}
        double t = t0 - 0.5 * dt;
        for (int64_t it = 1; it <= nt; ++it) {
            t += dt;
            update(h_loop, t);
            r = r + v * dt;
            rd = rd + vd * dt;
        }
        double t_final = d->t1;
        double dt_final = t_final - std::fma((double)nt - 0.5, dt, t0);
        update(d->q2m * 0.5 * dt_final, t_final);
        double* o = uN + 6 * i;
        double* od = duN + 6 * i;
        o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = v.x; o[4] = v.y; o[5] = v.z;
        od[0] = rd.x; od[1] = rd.y; od[2] = rd.z; od[3] = vd.x; od[4] = vd.y; od[5] = vd.z;
    }
    return TP_OK;
}

// Full-orbit ensemble (Boris, MultistepBoris, AdaptiveBoris, AdaptiveMultistepBoris).
int orc_boris_run(const tp_run_desc* d, const tp_field_desc* Ed, const tp_field_desc* Bd,
                  const orc_field_cb* Ecb, const orc_field_cb* Bcb, const orc_term_cb* tcb,
                  const double* u0, const double* dt_i, const double* tend_i, int64_t n,
                  int nthreads, int64_t nslots, double* t_out, double* u_out, int32_t* nsaved,
                  int8_t* retcode, int64_t* nsteps) {
    std::unique_ptr<Field> E = make_field(Ed, Ecb), B = make_field(Bd, Bcb);
    if (!E || !B) return TP_E_ARG;
    if (d->alg == TP_ALG_MULTISTEP || d->alg == TP_ALG_ADAPTIVE_MULTISTEP) {
        if (d->order != 2 && d->order != 4 && d->order != 6) return TP_E_ARG;
        if (d->nsub < 1) return TP_E_ARG;
    }
    if (d->savestepinterval < 1) return TP_E_ARG;
    Term term = make_term(&d->term, tcb);
    Params p{d->q2m, d->m, E.get(), B.get()};
    const int W = 6 + (d->save_fields ? 6 : 0) + (d->save_work ? 4 : 0);
    const int save_mask = (d->save_fields ? 1 : 0) | (d->save_work ? 2 : 0);
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    const bool multistep = d->alg == TP_ALG_MULTISTEP || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;

    // argument checks of every trajectory first (the reference throws before tracing)
    if (!adaptive) {
        for (int64_t i = 0; i < n; ++i) {
            double dt = dt_i ? dt_i[i] : d->dt;
            double t1 = tend_i ? tend_i[i] : d->t1;
            int64_t nt, nout;
            int st = orc_boris_counts(d->t0, t1, dt, d->maxiters, d->savestepinterval, d->save_start,
                                      d->save_end, d->save_everystep, &nt, &nout);
            if (st != TP_OK) return st;
        }
    }
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : overflow)
    for (int64_t i = 0; i < n; ++i) {
        Traj tr;
        double t1 = tend_i ? tend_i[i] : d->t1;
        const double* ui = u0 + 6 * i;
        if (!adaptive) {
            FixedOpts o;
            o.t0 = d->t0;
            o.t1 = t1;
            o.dt = dt_i ? dt_i[i] : d->dt;
            int64_t nt, nout;
            orc_boris_counts(d->t0, t1, o.dt, d->maxiters, d->savestepinterval, d->save_start,
                             d->save_end, d->save_everystep, &nt, &nout);
            o.nt = nt;
            o.nout = nout;
            o.ssi = d->savestepinterval;
            o.save_start = d->save_start != 0;
            o.save_end = d->save_end != 0;
            o.save_everystep = d->save_everystep != 0;
            o.save_fields = save_mask;
            if (multistep)
                boris_single(MultistepUpdater{d->order, d->nsub}, p, o, term, ui, tr);
            else
                boris_single(BorisUpdater{}, p, o, term, ui, tr);
        } else {
            if (multistep)
                adaptive_single(MultistepUpdater{d->order, d->nsub}, p, d->t0, t1, d->safety,
                                d->savestepinterval, d->save_start, d->save_end,
                                d->save_everystep, save_mask, d->step_cap, term, ui, tr);
            else
                adaptive_single(BorisUpdater{}, p, d->t0, t1, d->safety, d->savestepinterval,
                                d->save_start, d->save_end, d->save_everystep, save_mask,
                                d->step_cap, term, ui, tr);
        }
        if (!store(tr, i, n, W, nslots, t_out, u_out, nsaved, retcode, nsteps)) overflow |= 1;
    }
    return overflow ? TP_E_OVERFLOW : TP_OK;
}

// Detectors over packed trajectories (ext/TestParticleMeshesExt.jl:98-491).
// sums: nsurf x 4 (sum w, sum w v) accumulated trajectory after trajectory as
// the reference's get_particle_fluxes; counts: nsurf; rows (optional, sized by
// a counting call): surface-major (vx, vy, vz, w); first: n x 6 for surface 0.
int orc_detect(const double* t, const double* u, int32_t W, const int32_t* nsaved, int64_t n,
               const tp_surface* surf, int32_t nsurf, const double* weights, double weight, double* sums,
               int64_t* counts, double* rows, double* first) {
    std::vector<int64_t> off(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + std::max<int32_t>(nsaved[i], 0);
    if (sums)
        for (int64_t k = 0; k < (int64_t)nsurf * 4; ++k) sums[k] = 0.0;
    int64_t row = 0;
    for (int j = 0; j < nsurf; ++j) {
        int64_t cj = 0;
        for (int64_t i = 0; i < n; ++i) {
            const double w = weights ? weights[i] : weight;
            const double* ti = t + off[i];
            const double* ui = u + off[i] * W;
            det_walk(ti, ui, W, nsaved[i], surf[j], [&](const double* st) {
                cj += 1;
                if (sums) {
                    sums[4 * j] = sums[4 * j] + w;
                    for (int c = 0; c < 3; ++c) sums[4 * j + 1 + c] = sums[4 * j + 1 + c] + st[3 + c] * w;
                }
                if (rows) {
                    for (int c = 0; c < 3; ++c) rows[4 * row + c] = st[3 + c];
                    rows[4 * row + 3] = w;
                    row += 1;
                }
                return true;
            });
        }
        if (counts) counts[j] = cj;
    }
    if (first) {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        for (int64_t i = 0; i < n; ++i) {
            const double* ti = t + off[i];
            const double* ui = u + off[i] * W;
            double* o = first + 6 * i;
            for (int c = 0; c < 6; ++c) o[c] = nan;
            bool zero = false;
            bool done = false;
            det_walk(ti, ui, W, nsaved[i], surf[0], [&](const double* st) {
                if (!done) {
                    for (int c = 0; c < 6; ++c) o[c] = st[c];
                    done = true;
                }
                return false;
            }, &zero);
            if (zero)
                for (int c = 0; c < 6; ++c) o[c] = ui[c];
        }
    }
    return TP_OK;
}

// The hybrid's portable gyrophase trigonometry, for accuracy tests.
int orc_trig(const double* x, const double* y, int64_t n, double* s, double* c, double* a) {
    for (int64_t i = 0; i < n; ++i) {
        psincos(x[i], s[i], c[i]);
        a[i] = patan2(y[i], x[i]);
    }
    return TP_OK;
}

// Full orbit -> guiding centre -> full orbit (_get_gc_parameters then
// _gc_to_full, src/gc/gc.jl:13-39,128-154) for n states.
int orc_gc_roundtrip(const tp_field_desc* Ed, const tp_field_desc* Bd, const double* xv, int64_t n, double q,
                     double m, double t, double* out) {
    std::unique_ptr<Field> E = make_field(Ed, nullptr), B = make_field(Bd, nullptr);
    if (!E || !B) return TP_E_ARG;
    for (int64_t i = 0; i < n; ++i) {
        const double* s = xv + 6 * i;
        V3d X, x, v;
        double vpar, mu, phase;
        gc_params_phase({s[0], s[1], s[2]}, {s[3], s[4], s[5]}, *E, *B, q, m, t, X, vpar, mu, phase);
        GCState g{{X.x, X.y, X.z, vpar}};
        gc_to_full(g, *E, *B, q, m, mu, t, phase, x, v);
        double o[6] = {x.x, x.y, x.z, v.x, v.y, v.z};
        for (int c = 0; c < 6; ++c) out[6 * i + c] = o[c];
    }
    return TP_OK;
}

// Adaptive hybrid GC / full-orbit ensemble (src/hybrid.jl:234-474); the
// adiabaticity checks go to at_out / av_out when both are given.
int orc_hybrid_run(const tp_hybrid_desc* d, const tp_field_desc* Ed, const tp_field_desc* Bd,
                   const orc_field_cb* Ecb, const orc_field_cb* Bcb, const orc_term_cb* tcb, const double* u0,
                   int64_t n, int nthreads, int64_t nslots, int64_t aslots, double* t_out, double* u_out,
                   int32_t* nsaved, int8_t* retcode, int64_t* nsteps, double* at_out, double* av_out,
                   int32_t* nadia) {
    std::unique_ptr<Field> E = make_field(Ed, Ecb), B = make_field(Bd, Bcb);
    if (!E || !B) return TP_E_ARG;
    if (d->check_interval <= 0 || !(d->threshold_gc_to_fo >= d->threshold_fo_to_gc)) return TP_E_ARG;
    if (d->adiabaticity < TP_ADIA_CURVATURE || d->adiabaticity > TP_ADIA_JACOBIAN) return TP_E_ARG;
    if (d->savestepinterval < 1) return TP_E_ARG;
    Term term = make_term(&d->term, tcb);
    Params p{d->q2m, d->m, E.get(), B.get()};
    HybridOpts o;
    o.t0 = d->t0;
    o.t1 = d->t1;
    o.th_gc_fo = d->threshold_gc_to_fo;
    o.th_fo_gc = d->threshold_fo_to_gc;
    o.dtmin = d->dtmin;
    o.dtmax = d->dtmax;
    o.safety_fo = d->safety_fo;
    o.abstol = d->abstol;
    o.reltol = d->reltol;
    o.maxiters = d->maxiters;
    o.check = d->check_interval;
    o.ssi = d->savestepinterval;
    o.adia_mode = d->adiabaticity;
    o.save_start = d->save_start != 0;
    o.save_end = d->save_end != 0;
    o.save_everystep = d->save_everystep != 0;
    const bool want_adia = d->save_adiabaticity && at_out && av_out && nadia;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : overflow)
    for (int64_t i = 0; i < n; ++i) {
        HybridTraj h;
        hybrid_single(p, o, term, u0 + 6 * i, want_adia, h);
        if (!store(h.traj, i, n, 6, nslots, t_out, u_out, nsaved, retcode, nsteps)) overflow |= 1;
        if (want_adia) {
            int64_t na = (int64_t)h.at.size();
            nadia[i] = (int32_t)na;
            for (int64_t k = 0; k < std::min(na, aslots); ++k) {
                at_out[k * n + i] = h.at[k];
                av_out[(k * 2) * n + i] = h.av[2 * k];
                av_out[(k * 2 + 1) * n + i] = h.av[2 * k + 1];
            }
            if (na > aslots) overflow |= 1;
        }
    }
    return overflow ? TP_E_OVERFLOW : TP_OK;
}

// Guiding-centre ensemble (RK4 / RK45); per-particle q, q2m, mu optional.
int orc_gc_run(const tp_gc_desc* d, const tp_field_desc* Ed, const tp_field_desc* Bd,
               const orc_field_cb* Ecb, const orc_field_cb* Bcb, const orc_term_cb* tcb,
               const double* y0, const double* q_i, const double* q2m_i, const double* mu_i,
               const double* dt_i, const double* tend_i, int64_t n, int nthreads, int64_t nslots,
               double* t_out, double* u_out, int32_t* nsaved, int8_t* retcode, int64_t* nsteps) {
    std::unique_ptr<Field> E = make_field(Ed, Ecb), B = make_field(Bd, Bcb);
    if (!E || !B) return TP_E_ARG;
    Term term = make_term(&d->term, tcb);
    const int W = 4 + (d->save_fields ? 6 : 0) + (d->save_work ? 4 : 0);
    // _prepare_gc, src/gc/gc_solver.jl:187-231
    GCOpts o;
    o.t0 = d->t0;
    o.t1 = d->t1;
    o.dt = d->dt;
    o.dt_given = d->dt_given != 0;
    o.ssi = d->savestepinterval;
    o.maxiters = d->maxiters;
    o.save_start = d->save_start != 0;
    o.save_end = d->save_end != 0;
    o.save_everystep = d->save_everystep != 0;
    o.save_fields = (d->save_fields ? 1 : 0) | (d->save_work ? 2 : 0);
    o.abstol = d->abstol;
    o.reltol = d->reltol;
    double ttotal = d->t1 - d->t0;
    int64_t nt = 0;
    if (!o.dt_given) {
        if (d->alg == TP_GC_RK4) return TP_E_ARG;  // "dt must be provided for fixed step solver :rk4"
    } else {
        double sdt = (d->dt > 0) - (d->dt < 0), stt = (ttotal > 0) - (ttotal < 0);
        if (d->alg == TP_GC_RK4 && sdt != stt && ttotal != 0) return TP_E_ARG;
        nt = jl_round(ttotal / d->dt);
        if (d->alg == TP_GC_RK4 && nt > d->maxiters) nt = d->maxiters;
    }
    if (d->alg == TP_GC_RK4 && o.ssi < 1) return TP_E_ARG;
    int64_t nout = 0;
    if (o.save_start) nout += 1;
    if (d->alg == TP_GC_RK4 && o.save_everystep) {
        int64_t steps = nt / o.ssi;
        bool last_is_step = (nt > 0) && (nt % o.ssi == 0);
        nout += steps;
        if (!o.save_end && last_is_step) nout -= 1;
        if (o.save_end && !last_is_step) nout += 1;
    } else if (d->alg == TP_GC_RK4 && o.save_end) {
        nout += 1;
    }
    o.nt = nt;
    o.nout = nout;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(| : overflow)
    for (int64_t i = 0; i < n; ++i) {
        GCParams p{q_i ? q_i[i] : d->q, q2m_i ? q2m_i[i] : d->q2m, mu_i ? mu_i[i] : d->mu, E.get(),
                   B.get()};
        GCOpts oi = o;  // per-particle dt / tspan[2] (extension): _prepare_gc per particle
        if (dt_i || tend_i) {
            oi.dt = dt_i ? dt_i[i] : d->dt;
            oi.t1 = tend_i ? tend_i[i] : d->t1;
            if (d->alg == TP_GC_RK4) {
                int64_t nti = jl_round((oi.t1 - d->t0) / oi.dt);
                if (nti > d->maxiters) nti = d->maxiters;
                int64_t no = o.save_start ? 1 : 0;
                if (o.save_everystep) {
                    no += nti / o.ssi;
                    bool last_is_step = (nti > 0) && (nti % o.ssi == 0);
                    if (!o.save_end && last_is_step) no -= 1;
                    if (o.save_end && !last_is_step) no += 1;
                } else if (o.save_end) {
                    no += 1;
                }
                oi.nt = nti;
                oi.nout = no;
            } else if (dt_i) {
                oi.dt_given = true;
            }
        }
        Traj tr;
        if (d->alg == TP_GC_RK4)
            rk4_single(p, oi, term, y0 + 4 * i, tr);
        else
            rk45_single(p, oi, term, y0 + 4 * i, tr);
        if (!store(tr, i, n, W, nslots, t_out, u_out, nsaved, retcode, nsteps)) overflow |= 1;
    }
    return overflow ? TP_E_OVERFLOW : TP_OK;
}

// prepare_gc for n full-orbit states (src/gc/gc.jl:49-84)
int orc_gc_prepare(const tp_field_desc* Ed, const tp_field_desc* Bd, const orc_field_cb* Ecb,
                   const orc_field_cb* Bcb, const double* xv, int64_t n, double q, double m,
                   double t, double* y0_out, double* mu_out) {
    std::unique_ptr<Field> E = make_field(Ed, Ecb), B = make_field(Bd, Bcb);
    if (!E || !B) return TP_E_ARG;
    for (int64_t i = 0; i < n; ++i) {
        gc_parameters(xv + 6 * i, *E, *B, q, m, t, y0_out + 4 * i, y0_out + 4 * i + 3,
                      mu_out + i);
    }
    return TP_OK;
}

// gc_to_full (src/gc/gc.jl:106-154) at n guiding-centre states y (n x 4)
// with moments mu (n): xv_out (n x 6) at gyrophase phase_i[i] (or phase).
int orc_gc_to_full(const tp_field_desc* Ed, const tp_field_desc* Bd, const orc_field_cb* Ecb,
                   const orc_field_cb* Bcb, const double* y, const double* mu, int64_t n, double q,
                   double m, double phase, const double* phase_i, double t, double* xv_out) {
    std::unique_ptr<Field> E = make_field(Ed, Ecb), B = make_field(Bd, Bcb);
    if (!E || !B) return TP_E_ARG;
    for (int64_t i = 0; i < n; ++i) {
        GCState s{{y[4 * i], y[4 * i + 1], y[4 * i + 2], y[4 * i + 3]}};
        V3d x, v;
        gc_to_full(s, *E, *B, q, m, mu[i], t, phase_i ? phase_i[i] : phase, x, v);
        double* o = xv_out + 6 * i;
        o[0] = x.x;
        o[1] = x.y;
        o[2] = x.z;
        o[3] = v.x;
        o[4] = v.y;
        o[5] = v.z;
    }
    return TP_OK;
}

// Field values (and optionally Jacobians, row-major 9 per point) at n points.
int orc_field_eval(const tp_field_desc* d, const orc_field_cb* cb, const double* x, int64_t n,
                   double t, double* out, double* jac_out) {
    std::unique_ptr<Field> F = make_field(d, cb);
    if (!F) return TP_E_ARG;
    for (int64_t i = 0; i < n; ++i) {
        V3d r{x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        if (jac_out) {
            V3d v;
            M3 J;
            F->jac(r, t, v, J);
            out[3 * i] = v.x;
            out[3 * i + 1] = v.y;
            out[3 * i + 2] = v.z;
            std::memcpy(jac_out + 9 * i, J.a, sizeof(J.a));
        } else {
            V3d v = F->eval(r, t);
            out[3 * i] = v.x;
            out[3 * i + 1] = v.y;
            out[3 * i + 2] = v.z;
        }
    }
    return TP_OK;
}

}  // extern "C"
