// noalloc.cu -- tp_pack_results_device_noalloc: result packing that allocates nothing.
//
// Who needs it: callers that own every byte of device memory and forbid a
// library from calling cudaMalloc / cudaMallocAsync -- a host framework with
// its own memory pool (a Julia or Python runtime that hands out all buffers),
// a serving process with a fixed memory budget, or code that must not hit the
// allocator on its latency path.  They run the push with tp_boris_run_device
// into their own buffers; this entry point then turns the slot-major output
// into the reference's per-trajectory packed layout.  The scan it needs (one
// offset per trajectory plus per-block partial sums) lives in a file-scope
// __device__ array instead of an allocated buffer.
//
// Limits and sharing.  The array holds TP_NOALLOC_MAX_TRAJECTORIES + 1
// offsets and one partial sum per 1024 trajectories (about 8.4 MB); every GPU
// that loads the library keeps it until the process exits.  Larger n is
// rejected with TP_E_ARG.  All calls share the one array: every element a call
// reads is first written by that same call (nothing accumulates across calls,
// so nothing needs clearing), but two calls whose kernels overlap on the GPU --
// on two streams, or from two host threads -- race on it and must not be
// issued.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture begins.  The address is cached per device for the
// life of the process: it is valid until the device's primary context is
// destroyed (cudaDeviceReset), after which the library must not be called.
// Counts are clamped to [0, nslots], as the allocating path does (pack.cu).
#include <cub/block/block_scan.cuh>

#include <cstring>
#include <mutex>
#include <string>

#include "tp_launch.h"

namespace tpb {

namespace {

constexpr int kBlock = 1024;
constexpr int64_t kMax = TP_NOALLOC_MAX_TRAJECTORIES;
constexpr int64_t kMaxBlocks = (kMax + kBlock - 1) / kBlock;

// offsets[0 .. kMax] then block sums[0 .. kMaxBlocks] (the last one is the total)
static __device__ __align__(256) int64_t g_noalloc_scratch[kMax + 1 + kMaxBlocks + 1];

std::mutex g_setup_mu;
int64_t* g_scratch_ptr[64] = {nullptr};

// per-block exclusive prefix of clamp(nsaved, 0, nslots); block totals
__global__ void __launch_bounds__(kBlock) k_na_block_scan(const int32_t* nsaved, int64_t n, int64_t nslots,
                                                          int64_t* scratch) {
    typedef cub::BlockScan<int64_t, kBlock> Scan;
    __shared__ typename Scan::TempStorage tmp;
    int64_t* offsets = scratch;
    int64_t* bsum = scratch + kMax + 1;
    int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    int64_t c = 0;
    if (i < n) {
        c = nsaved[i];
        c = c < 0 ? 0 : (c > nslots ? nslots : c);
    }
    int64_t excl, total;
    Scan(tmp).ExclusiveSum(c, excl, total);
    if (i < n) offsets[i] = excl;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// exclusive scan of the block totals (at most kMaxBlocks = 1024 of them)
__global__ void __launch_bounds__(kBlock) k_na_scan_blocks(int64_t nblocks, int64_t* scratch, int64_t* total_out) {
    typedef cub::BlockScan<int64_t, kBlock> Scan;
    __shared__ typename Scan::TempStorage tmp;
    int64_t* bsum = scratch + kMax + 1;
    int64_t v = threadIdx.x < nblocks ? bsum[threadIdx.x] : 0;
    int64_t excl, total;
    Scan(tmp).ExclusiveSum(v, excl, total);
    __syncthreads();
    if (threadIdx.x < nblocks) bsum[threadIdx.x] = excl;
    if (threadIdx.x == 0) {
        bsum[kMaxBlocks] = total;
        if (total_out) *total_out = total;
    }
}

// slot-major -> packed, trajectory i at offset (block prefix + in-block prefix)
__global__ void k_na_pack(const double* t_in, const double* u_in, const int32_t* nsaved, int64_t n,
                          int64_t nslots, int W, const int64_t* scratch, double* t_out, double* u_out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t* offsets = scratch;
    const int64_t* bsum = scratch + kMax + 1;
    int64_t ns = nsaved[i];
    ns = ns < 0 ? 0 : (ns > nslots ? nslots : ns);
    int64_t o = bsum[i / kBlock] + offsets[i];
    for (int64_t k = 0; k < ns; ++k) {
        t_out[o + k] = t_in[k * n + i];
        for (int c = 0; c < W; ++c) u_out[(o + k) * W + c] = u_in[(k * W + c) * n + i];
    }
}

}  // namespace

// Device address of the static scratch for the current device (looked up once).
int noalloc_scratch(int device, int64_t** out) {
    if (device < 0 || device >= 64) return TP_E_ARG;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return TP_E_CUDA;
        g_scratch_ptr[device] = static_cast<int64_t*>(p);
    }
    *out = g_scratch_ptr[device];
    return TP_OK;
}

cudaError_t launch_noalloc_pack(int64_t* scratch, const double* t_in, const double* u_in,
                                const int32_t* nsaved, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, int64_t* total_out, cudaStream_t s) {
    int64_t nblocks = (n + kBlock - 1) / kBlock;
    if (nblocks < 1) nblocks = 1;
    k_na_block_scan<<<(unsigned)nblocks, kBlock, 0, s>>>(nsaved, n, nslots, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_na_scan_blocks<<<1, kBlock, 0, s>>>(nblocks, scratch, total_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int pb = 128;
    k_na_pack<<<(unsigned)((n + pb - 1) / pb), pb, 0, s>>>(t_in, u_in, nsaved, n, nslots, width, scratch,
                                                          t_out, u_out);
    return cudaGetLastError();
}

}  // namespace tpb

// ============================================================== C ABI
extern "C" int tp_pack_results_device_noalloc(tp_ctx* ctx, const double* t_in, const double* u_in,
                                              const int32_t* nsaved, int64_t n, int64_t nslots,
                                              int32_t width, double* t_out, double* u_out,
                                              int64_t* total_out, void* stream) {
    using namespace tpb;
    if (!ctx) return TP_E_ARG;
    if (n < 0 || nslots < 0 || width < 1) return ctx_fail(ctx, TP_E_ARG, "negative size or width < 1");
    if (n > TP_NOALLOC_MAX_TRAJECTORIES)
        return ctx_fail(ctx, TP_E_ARG,
                        "tp_pack_results_device_noalloc: n = " + std::to_string(n) +
                            " exceeds the static scratch limit of " +
                            std::to_string((long long)TP_NOALLOC_MAX_TRAJECTORIES) + " trajectories");
    if (!nsaved || !total_out || (n > 0 && nslots > 0 && (!t_in || !u_in || !t_out || !u_out)))
        return ctx_fail(ctx, TP_E_ARG, "null device buffer");
    int dev = ctx_device(ctx), prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return ctx_fail(ctx, TP_E_CUDA, "cudaSetDevice failed");
    int64_t* scratch = nullptr;
    int st = noalloc_scratch(dev, &scratch);
    cudaError_t e = cudaSuccess;
    cudaStream_t s = (cudaStream_t)stream;
    if (st == TP_OK) {
        if (n == 0)
            e = cudaMemsetAsync(total_out, 0, sizeof(int64_t), s);
        else
            e = launch_noalloc_pack(scratch, t_in, u_in, nsaved, n, nslots, width, t_out, u_out, total_out, s);
    }
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    if (st != TP_OK) return ctx_fail(ctx, st, "cudaGetSymbolAddress of the static scratch failed");
    if (e != cudaSuccess) return ctx_fail(ctx, TP_E_CUDA, std::string("noalloc pack: ") + cudaGetErrorString(e));
    return TP_OK;
}
