// gc_fp64.cu -- float64 guiding-centre kernels (the drop-in path) and the
// prepare_gc kernel.  Compiled with -fmad=false (see fields64.cuh).
#include "gc_common.cuh"

namespace tpb {

// _get_gc_parameters (src/gc/gc.jl:13-39) for one full-orbit state:
// X = x - rho, v_par, mu in the E x B frame.
__global__ void k_gc_prepare(GCPrepArgs a) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double* s = a.xv + 6 * i;
    D3 x{s[0], s[1], s[2]}, v{s[3], s[4], s[5]};
    D3 bp = field_eval64(a.f.B, x, a.t);
    double Bmp = norm(bp);
    D3 bhp = bp / Bmp;
    D3 rho = cross(bhp, v) / (a.q / a.m * Bmp);
    D3 X = x - rho;
    D3 b = field_eval64(a.f.B, X, a.t);
    double Bmag = norm(b);
    D3 bh = b / Bmag;
    double vpar = dot(bh, v);
    D3 vperp = v - vpar * bh;
    D3 e = field_eval64(a.f.E, X, a.t);
    D3 vE = cross(e, bh) / Bmag;
    D3 w = vperp - vE;
    double mu = a.m * dot(w, w) / (2.0 * Bmag);
    a.y0[4 * i + 0] = X.x;
    a.y0[4 * i + 1] = X.y;
    a.y0[4 * i + 2] = X.z;
    a.y0[4 * i + 3] = vpar;
    a.mu[i] = mu;
}

cudaError_t launch_gc_prepare(const GCPrepArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    int block = 256;
    int64_t grid = (a.n + block - 1) / block;
    k_gc_prepare<<<(unsigned)grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

// get_fields / get_work (src/boris/boris.jl:599-640) at n states: E and B,
// then the work rates of get_work_rates (src/equations.jl:394-441) or
// get_work_rates_gc (:445-480), in the order of the savers.
__global__ void k_eval_points(PointsArgs a) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double* s = a.u + (int64_t)a.stride * i;
    const double t = a.t[i];
    double* o = a.out + (int64_t)a.wout * i;
    D3 x{s[0], s[1], s[2]};
    int c = 0;
    if (a.want & 1) {
        D3 E = field_eval64(a.f.E, x, t), B = field_eval64(a.f.B, x, t);
        o[0] = E.x;
        o[1] = E.y;
        o[2] = E.z;
        o[3] = B.x;
        o[4] = B.y;
        o[5] = B.z;
        c = 6;
    }
    if (a.want & 2) {
        double W[4];
        const double q2m = a.q2m_i ? a.q2m_i[i] : a.q2m;
        if (a.kind == TP_POINTS_GC)
            work_rates_gc64<GM_ANY>(a.f, x, s[3], t, a.q_i ? a.q_i[i] : a.q, q2m, a.mu_i ? a.mu_i[i] : a.mu, W);
        else
            work_rates64<GM_ANY>(a.f, x, D3{s[3], s[4], s[5]}, t, q2m, a.m_i ? a.m_i[i] : a.m, W);
        for (int k = 0; k < 4; ++k) o[c + k] = W[k];
    }
}

// save_work columns (_prepare_saved_data, src/boris/boris.jl:429-437;
// gc_solver.jl:233-248): the work rates of every saved state, one thread per
// (slot, particle), written after the push so the push kernels carry no
// Jacobian code
__global__ void k_fill_work(WorkFillArgs a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.nslots * a.n) return;
    const int64_t k = idx / a.n, i = idx - k * a.n;
    if (k >= a.nsaved[i]) return;
    const int64_t n = a.n;
    double* u = a.u_out + (k * a.W) * n + i;
    const double t = a.t_out[k * n + i];
    const D3 x{u[0], u[n], u[2 * n]};
    double W[4];
    if (a.gc) {
        const double q = a.q_i ? a.q_i[i] : a.q;
        const double q2m = a.q2m_i ? a.q2m_i[i] : a.q2m;
        const double mu = a.mu_i ? a.mu_i[i] : a.mu;
        work_rates_gc64<GM_ANY>(a.f, x, u[3 * n], t, q, q2m, mu, W);
    } else {
        work_rates64<GM_ANY>(a.f, x, D3{u[3 * n], u[4 * n], u[5 * n]}, t, a.q2m, a.m, W);
    }
    for (int c = 0; c < 4; ++c) u[(int64_t)(a.c0 + c) * n] = W[c];
}

cudaError_t launch_fill_work(const WorkFillArgs& a, cudaStream_t s) {
    const int64_t total = a.nslots * a.n;
    if (total <= 0) return cudaSuccess;
    const int block = 128;
    k_fill_work<<<(unsigned)((total + block - 1) / block), block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_eval_points(const PointsArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    int block = 128;
    int64_t grid = (a.n + block - 1) / block;
    k_eval_points<<<(unsigned)grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <class R>
static const void* gc_kernel(bool rk4, bool queue) {
    if (rk4) return queue ? (const void*)k_rk4<R, true> : (const void*)k_rk4<R, false>;
    return queue ? (const void*)k_rk45<R, true> : (const void*)k_rk45<R, false>;
}

const void* select_gc_kernel64(const GCArgs& a, bool queue) {
    const int gm = gc_grid_mode(a.f);
    bool rk4 = a.alg == TP_GC_RK4;
    if (gm == GM_ANY) return gc_kernel<RHS64<GM_ANY>>(rk4, queue);
    return gm == GM_GRID ? gc_kernel<RHS64<GM_GRID>>(rk4, queue) : gc_kernel<RHS64<GM_ANALYTIC>>(rk4, queue);
}

const void* select_gc_kernel32(const GCArgs& a, bool queue);

cudaError_t prime_gc(const GCArgs& a) {
    const bool q = a.use_queue != 0;
    cudaFuncAttributes at;
    return cudaFuncGetAttributes(&at, a.precision == TP_GC_PREC_FP32RHS ? select_gc_kernel32(a, q)
                                                                         : select_gc_kernel64(a, q));
}

cudaError_t prime_fill_work() {
    cudaFuncAttributes at;
    return cudaFuncGetAttributes(&at, (const void*)k_fill_work);
}

int occupancy_gc(const GCArgs& a, int block) {
    int nb = 0;
    const void* f = a.precision == TP_GC_PREC_FP32RHS ? select_gc_kernel32(a, true) : select_gc_kernel64(a, true);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, block, 0);
    return nb;
}

cudaError_t launch_gc(const GCArgs& a, const LaunchCfg& c, cudaStream_t s) {
    const bool q = a.use_queue != 0;
    const void* f = a.precision == TP_GC_PREC_FP32RHS ? select_gc_kernel32(a, q) : select_gc_kernel64(a, q);
    void* args[] = {const_cast<GCArgs*>(&a)};
    return cudaLaunchKernel(f, dim3(c.grid), dim3(c.block), args, 0, s);
}

}  // namespace tpb
