// pack.cu -- layout kernels: field node tables and result packing.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "tp_launch.h"

namespace tpb {

// (3, nx, ny, nz) column-major source -> 4-vector per node table, entry
// node*stride + off (stride 2 interleaves E and B of one node in 32 bytes).
template <class S, class D>
__global__ void k_pack_nodes(const S* src, int64_t nodes, D* dst, int stride, int off) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    D* o = dst + 4 * (k * stride + off);
    o[0] = (D)src[3 * k + 0];
    o[1] = (D)src[3 * k + 1];
    o[2] = (D)src[3 * k + 2];
    o[3] = (D)0;
}

cudaError_t launch_pack_node_table(const void* src, int src_f64, int64_t nodes, void* dst,
                                   int dst_f64, int stride, int off, cudaStream_t s) {
    if (nodes <= 0) return cudaSuccess;
    const int block = 256;
    const unsigned grid = (unsigned)((nodes + block - 1) / block);
    if (src_f64 && dst_f64)
        k_pack_nodes<double, double><<<grid, block, 0, s>>>((const double*)src, nodes, (double*)dst, stride, off);
    else if (src_f64)
        k_pack_nodes<double, float><<<grid, block, 0, s>>>((const double*)src, nodes, (float*)dst, stride, off);
    else if (dst_f64)
        k_pack_nodes<float, double><<<grid, block, 0, s>>>((const float*)src, nodes, (double*)dst, stride, off);
    else
        k_pack_nodes<float, float><<<grid, block, 0, s>>>((const float*)src, nodes, (float*)dst, stride, off);
    return cudaGetLastError();
}

// slot-major (t[k*n+i], u[(k*W+c)*n+i]) -> per-trajectory packed
// (t_out[off_i + k], u_out[(off_i + k)*W + c]).  One warp per particle
// group: threads stride over (particle, save) pairs.
__global__ void k_pack_results(const double* t_in, const double* u_in, const int32_t* nsaved,
                               const int64_t* offsets, int64_t n, int64_t nslots, int W,
                               double* t_out, double* u_out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t ns = nsaved[i];
    ns = ns < 0 ? 0 : (ns > nslots ? nslots : ns);
    int64_t o = offsets[i];
    for (int64_t k = 0; k < ns; ++k) {
        t_out[o + k] = t_in[k * n + i];
        for (int c = 0; c < W; ++c) u_out[(o + k) * W + c] = u_in[(k * W + c) * n + i];
    }
}

cudaError_t launch_pack_results(const double* t_in, const double* u_in, const int32_t* nsaved,
                                const int64_t* offsets, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int block = 128;
    const unsigned grid = (unsigned)((n + block - 1) / block);
    k_pack_results<<<grid, block, 0, s>>>(t_in, u_in, nsaved, offsets, n, nslots, width, t_out, u_out);
    return cudaGetLastError();
}

// nsaved (clamped to [0, nslots]) -> exclusive offsets, plus the total in offsets[n]
__global__ void k_clamp_counts(const int32_t* nsaved, int64_t n, int64_t nslots, int64_t* cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        cnt[n] = 0;
        return;
    }
    int64_t v = nsaved[i];
    cnt[i] = v < 0 ? 0 : (v > nslots ? nslots : v);
}

cudaError_t scan_offsets(const int32_t* nsaved, int64_t n, int64_t nslots, int64_t* cnt,
                         int64_t* offsets, void* tmp, size_t* tmp_bytes, cudaStream_t s) {
    if (!tmp) {
        return cub::DeviceScan::ExclusiveSum(nullptr, *tmp_bytes, cnt, offsets, n + 1, s);
    }
    const int block = 256;
    k_clamp_counts<<<(unsigned)((n + 1 + block - 1) / block), block, 0, s>>>(nsaved, n, nslots, cnt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cub::DeviceScan::ExclusiveSum(tmp, *tmp_bytes, cnt, offsets, n + 1, s);
}

// ---------------------------------------------------------------- cell ordering
// Morton (Z-order) key of each particle's initial cell on grid g: 10 bits per
// axis of the cell index (coarsened on axes of more than 1024 cells), so
// particles sorted by key lie in compact 3-D blocks of cells.
__device__ __forceinline__ uint32_t spread10(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void k_cell_keys(const double* u0, int64_t n, DevField g, uint32_t* keys, int32_t* idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[3];
    for (int a = 0; a < 3; ++a) {
        const double u = (u0[6 * i + a] - g.x0[a]) * g.inv_dx[a];
        const int64_t na = g.n[a] > 0 ? g.n[a] : 1;
        int64_t k = isfinite(u) ? (int64_t)floor(fmin(fmax(u, -4.0e18), 4.0e18)) : 0;
        k %= na;
        if (k < 0) k += na;
        int sh = 0;
        while ((na - 1) >> (10 + sh)) ++sh;
        c[a] = (uint32_t)(k >> sh);
    }
    keys[i] = spread10(c[0]) | (spread10(c[1]) << 1) | (spread10(c[2]) << 2);
    idx[i] = (int32_t)i;
}

// perm = the particles ordered by the Morton key of their initial cell on g;
// tmp: scratch of tmp_bytes (first call with tmp = null sizes it: 2 n keys,
// 2 n indices and the radix sort's own storage)
cudaError_t cell_order(const double* u0, int64_t n, const DevField& g, void* tmp, size_t* tmp_bytes,
                       int32_t** perm, cudaStream_t s) {
    const size_t kb = ((size_t)n * sizeof(uint32_t) + 255) & ~(size_t)255;
    const size_t ib = ((size_t)n * sizeof(int32_t) + 255) & ~(size_t)255;
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, 30, s);
    if (!tmp) {
        *tmp_bytes = 2 * kb + 2 * ib + sort_bytes;
        return cudaSuccess;
    }
    char* b = static_cast<char*>(tmp);
    uint32_t* k_in = reinterpret_cast<uint32_t*>(b);
    uint32_t* k_out = reinterpret_cast<uint32_t*>(b + kb);
    int32_t* v_in = reinterpret_cast<int32_t*>(b + 2 * kb);
    int32_t* v_out = reinterpret_cast<int32_t*>(b + 2 * kb + ib);
    void* st = b + 2 * kb + 2 * ib;
    const int block = 256;
    k_cell_keys<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(u0, n, g, k_in, v_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortPairs(st, sort_bytes, k_in, k_out, v_in, v_out, (int)n, 0, 30, s);
    *perm = v_out;
    return e;
}

}  // namespace tpb
