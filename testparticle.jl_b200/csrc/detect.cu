// detect.cu -- virtual detectors over packed trajectories: surface crossings,
// particle fluxes and first crossings (get_particle_crossings,
// get_particle_flux(es), get_first_crossing; ext/TestParticleMeshesExt.jl:98-491).
//
// One thread per trajectory walks its saves in time order, so the crossings
// of a trajectory are found, and its partial sums accumulated, in the
// reference's order.  Per-surface totals are then reduced over trajectories
// in a fixed order by one block per surface (deterministic run to run).
// Compiled with -fmad=false: distances, crossing fractions and the linear
// interpolation follow the CPU restatement operation for operation; the
// crossing time is fma(f, t2 - t1, t1), the reference's muladd.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "fields64.cuh"
#include "tp_launch.h"

namespace tpb {

namespace {

struct DetArgs {
    const double* t;
    const double* u;
    const int32_t* nsaved;
    const int64_t* off;     // n + 1 trajectory offsets
    int64_t n;
    int32_t width, nsurf;
    const tp_surface* surf; // device copy
    const double* weights;  // n, or null
    double weight;
    int64_t* cnt;           // nsurf x n crossing counts (count pass)
    double* part;           // nsurf x n x 4 partial sums (flux pass), or null
    const int64_t* roff;    // nsurf x n + 1 row offsets (row pass)
    double* rows;           // total x 4 (row pass)
    double* first;          // n x 6 (first-crossing pass)
};

__device__ __forceinline__ double sdist(const tp_surface& S, D3 p) {
    D3 v = p - D3{S.point[0], S.point[1], S.point[2]};
    if (S.kind == TP_SURF_SPHERE) return norm(v) - S.radius;
    return dot(v, D3{S.normal[0], S.normal[1], S.normal[2]});
}

__device__ __forceinline__ bool valid(const tp_surface& S, D3 p) {
    if (S.kind != TP_SURF_DISK) return true;
    D3 d = p - D3{S.point[0], S.point[1], S.point[2]};
    return dot(d, d) <= S.radius * S.radius;
}

__device__ __forceinline__ D3 pos(const DetArgs& a, int64_t row) {
    const double* r = a.u + row * a.width;
    return {r[0], r[1], r[2]};
}

// the trajectory's state at time tc: searchsortedlast over its save times,
// then u_i + theta (u_{i+1} - u_i) (clamped to the first / last save)
__device__ __forceinline__ void interp(const DetArgs& a, int64_t o, int64_t m, double tc, double s[6]) {
    int64_t lo = 0, hi = m;  // first index with t > tc
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a.t[o + mid] <= tc) lo = mid + 1;
        else hi = mid;
    }
    const int64_t i = lo - 1;  // searchsortedlast (0-based), -1 if none
    if (i < 0 || i >= m - 1) {
        const double* r = a.u + (o + (i < 0 ? 0 : m - 1)) * a.width;
        for (int c = 0; c < 6; ++c) s[c] = r[c];
        return;
    }
    const double th = (tc - a.t[o + i]) / (a.t[o + i + 1] - a.t[o + i]);
    const double* r0 = a.u + (o + i) * a.width;
    const double* r1 = r0 + a.width;
    for (int c = 0; c < 6; ++c) s[c] = r0[c] + th * (r1[c] - r0[c]);
}

// walk trajectory i for surface S; MODE 0 count (+ partial sums), 1 rows, 2 first crossing
template <int MODE>
__device__ __forceinline__ void walk(const DetArgs& a, int64_t i, int j, const tp_surface& S) {
    const int64_t o = a.off[i], m = a.nsaved[i];
    const double w = a.weights ? a.weights[i] : a.weight;
    int64_t count = 0;
    double sw = 0.0, sv[3] = {0.0, 0.0, 0.0};
    int64_t r = (MODE == 1) ? a.roff[(int64_t)j * a.n + i] : 0;
    bool found = false;
    if (m >= 1) {
        D3 p1 = pos(a, o);
        double s1 = sdist(S, p1);
        if (MODE == 2 && s1 == 0.0) {
            for (int c = 0; c < 6; ++c) a.first[6 * i + c] = a.u[o * a.width + c];
            return;
        }
        for (int64_t k = 0; k + 1 < m; ++k) {
            D3 p2 = pos(a, o + k + 1);
            double s2 = sdist(S, p2);
            if (s1 * s2 < 0.0 || (s1 != 0.0 && s2 == 0.0)) {
                double f = s1 / (s1 - s2);
                D3 pc = p1 + f * (p2 - p1);
                if (valid(S, pc)) {
                    double tl = a.t[o + k], tr = a.t[o + k + 1];
                    double tc = fma(f, tr - tl, tl);
                    double st[6];
                    interp(a, o, m, tc, st);
                    if (MODE == 2) {
                        for (int c = 0; c < 6; ++c) a.first[6 * i + c] = st[c];
                        found = true;
                        break;
                    }
                    if (MODE == 1) {
                        double* row = a.rows + 4 * r;
                        row[0] = st[3];
                        row[1] = st[4];
                        row[2] = st[5];
                        row[3] = w;
                        r += 1;
                    } else {
                        count += 1;
                        sw = sw + w;
                        for (int c = 0; c < 3; ++c) sv[c] = sv[c] + st[3 + c] * w;
                    }
                }
            }
            s1 = s2;
            p1 = p2;
        }
    }
    if (MODE == 2) {
        if (!found) {
            const double q = __longlong_as_double(0x7ff8000000000000ULL);
            for (int c = 0; c < 6; ++c) a.first[6 * i + c] = q;
        }
        return;
    }
    if (MODE == 0) {
        const int64_t idx = (int64_t)j * a.n + i;
        a.cnt[idx] = count;
        if (a.part) {
            a.part[4 * idx + 0] = sw;
            a.part[4 * idx + 1] = sv[0];
            a.part[4 * idx + 2] = sv[1];
            a.part[4 * idx + 3] = sv[2];
        }
    }
}

template <int MODE>
__global__ void k_detect(DetArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    for (int j = 0; j < a.nsurf; ++j) {
        const tp_surface S = a.surf[j];
        walk<MODE>(a, i, j, S);
    }
}

// per-surface totals of the partial sums, fixed order: thread k sums the
// trajectories k, k + 256, ... in order, then a tree over the 256 threads
constexpr int kRedThreads = 256;
__global__ void __launch_bounds__(kRedThreads) k_det_reduce(const double* part, int64_t n, double* tot) {
    __shared__ double sh[4][kRedThreads];
    const int j = blockIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = threadIdx.x; i < n; i += kRedThreads)
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + part[4 * ((int64_t)j * n + i) + c];
    for (int c = 0; c < 4; ++c) sh[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = kRedThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int c = 0; c < 4; ++c) sh[c][threadIdx.x] = sh[c][threadIdx.x] + sh[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; ++c) tot[4 * j + c] = sh[c][0];
}

__global__ void k_widen(const int32_t* in, int64_t n, int64_t* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) out[i] = (i < n) ? (int64_t)(in[i] < 0 ? 0 : in[i]) : 0;
}

}  // namespace

// exclusive scan of int64 counts (length m + 1, the last entry 0)
static cudaError_t scan64(const int64_t* in, int64_t m1, int64_t* out, cudaStream_t s) {
    size_t bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, m1, s);
    if (e != cudaSuccess) return e;
    void* tmp = nullptr;
    e = cudaMallocAsync(&tmp, bytes, s);
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, m1, s);
    cudaFreeAsync(tmp, s);
    return e;
}

// mode 0: fluxes (tot: nsurf x 4), 1: crossings (counts, rows), 2: first crossing
cudaError_t launch_detect(int mode, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                          int64_t n, const tp_surface* surf_d, int32_t nsurf, const double* weights,
                          double weight, double* tot, int64_t* counts_h, double** rows_d_out, double* first,
                          cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    int64_t *off = nullptr, *wide = nullptr, *cnt = nullptr, *roff = nullptr;
    double* part = nullptr;
    const int block = 128;
    const unsigned grid = (unsigned)((n + block - 1) / block);
    e = cudaMallocAsync((void**)&wide, (size_t)(n + 1) * sizeof(int64_t), s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&off, (size_t)(n + 1) * sizeof(int64_t), s);
    if (e == cudaSuccess) {
        k_widen<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(nsaved, n, wide);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = scan64(wide, n + 1, off, s);
    DetArgs a;
    memset(&a, 0, sizeof(a));
    a.t = t;
    a.u = u;
    a.nsaved = nsaved;
    a.off = off;
    a.n = n;
    a.width = width;
    a.nsurf = nsurf;
    a.surf = surf_d;
    a.weights = weights;
    a.weight = weight;
    a.first = first;
    if (e == cudaSuccess && mode == 2) {
        k_detect<2><<<grid, block, 0, s>>>(a);
        e = cudaGetLastError();
    }
    const int64_t m = (int64_t)nsurf * n;
    if (e == cudaSuccess && mode != 2) e = cudaMallocAsync((void**)&cnt, (size_t)(m + 1) * sizeof(int64_t), s);
    if (e == cudaSuccess && mode == 0) e = cudaMallocAsync((void**)&part, (size_t)std::max<int64_t>(m, 1) * 4 * sizeof(double), s);
    if (e == cudaSuccess && mode != 2) {
        a.cnt = cnt;
        a.part = part;
        e = cudaMemsetAsync(cnt + m, 0, sizeof(int64_t), s);
        if (e == cudaSuccess) {
            k_detect<0><<<grid, block, 0, s>>>(a);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && mode == 0) {
        k_det_reduce<<<(unsigned)nsurf, kRedThreads, 0, s>>>(part, n, tot);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && mode == 1) {
        e = cudaMallocAsync((void**)&roff, (size_t)(m + 1) * sizeof(int64_t), s);
        if (e == cudaSuccess) e = scan64(cnt, m + 1, roff, s);
        // per-surface counts: the row offsets at the surface boundaries
        std::vector<int64_t> bnd(nsurf + 1);
        for (int j = 0; j <= nsurf && e == cudaSuccess; ++j)
            e = cudaMemcpyAsync(&bnd[j], roff + (int64_t)j * n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) {
            for (int j = 0; j < nsurf; ++j) counts_h[j] = bnd[j + 1] - bnd[j];
            const int64_t total = bnd[nsurf];
            if (rows_d_out) {
                double* rows = nullptr;
                e = cudaMallocAsync((void**)&rows, (size_t)std::max<int64_t>(total, 1) * 4 * sizeof(double), s);
                if (e == cudaSuccess) {
                    a.roff = roff;
                    a.rows = rows;
                    k_detect<1><<<grid, block, 0, s>>>(a);
                    e = cudaGetLastError();
                }
                *rows_d_out = rows;
            }
        }
    }
    for (void* q : {(void*)off, (void*)wide, (void*)cnt, (void*)roff, (void*)part})
        if (q) cudaFreeAsync(q, s);
    return e;
}

}  // namespace tpb
