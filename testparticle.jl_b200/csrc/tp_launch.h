// tp_launch.h -- internal launcher declarations shared by the kernel
// translation units and the runtime (not part of the public C ABI).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "tp_device.cuh"

namespace tpb {

struct LaunchCfg {
    int grid;
    int block;
};

// guiding-centre launch block
struct GCArgs {
    DevFields f;
    DevTerm term;
    int32_t alg, precision, save_fields, dt_given;
    int32_t save_start, save_end, save_everystep, pad;
    double t0, t1, dt, q, q2m, mu, abstol, reltol;
    int64_t ssi, maxiters, nt, nout;
    int64_t n, nslots;
    const double* y0;     // 4 x n
    const double* q_i;    // optional per-particle
    const double* q2m_i;
    const double* mu_i;
    const double* dt_i;   // optional per-particle dt
    const double* tend_i; // optional per-particle tspan[2]
    double* t_out;        // nslots x n
    double* u_out;        // nslots x W x n
    int32_t* nsaved;
    int8_t* retcode;
    int64_t* nsteps;
    int32_t* status;
    unsigned long long* queue;
    int32_t use_queue;
    int32_t pad2;
    uint64_t budget_ns;
};

struct GCPrepArgs {
    DevFields f;
    const double* xv;
    int64_t n;
    double q, m, t;
    double* y0;
    double* mu;
};

cudaError_t launch_boris_fp64(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_boris_fp32c(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s);
int occupancy_boris_fp64(const BorisArgs& a, int block);
int occupancy_boris_fp32c(const BorisArgs& a, int block);

cudaError_t launch_gc(const GCArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_gc_fp32(const GCArgs& a, const LaunchCfg& c, cudaStream_t s);
int occupancy_gc(const GCArgs& a, int block);
cudaError_t launch_gc_prepare(const GCPrepArgs& a, cudaStream_t s);

// context accessors for translation units outside runtime.cu
int ctx_device(const tp_ctx* ctx);
int ctx_fail(tp_ctx* ctx, int code, const std::string& msg);

// static-scratch packing (noalloc.cu)
int noalloc_scratch(int device, int64_t** out);
cudaError_t launch_noalloc_pack(int64_t* scratch, const double* t_in, const double* u_in,
                                const int32_t* nsaved, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, int64_t* total_out, cudaStream_t s);

// packing helpers (pack.cu)
cudaError_t launch_pack_node_table(const void* src, int src_f64, int64_t nodes, void* dst,
                                   int dst_f64, int stride, int off, cudaStream_t s);
cudaError_t launch_pack_results(const double* t_in, const double* u_in, const int32_t* nsaved,
                                const int64_t* offsets, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, cudaStream_t s);

}  // namespace tpb
