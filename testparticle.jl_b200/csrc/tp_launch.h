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
    int32_t save_work;    // work rates appended to every save (width + 4)
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

// gc_to_full at n guiding-centre states (y: n x 4, mu: n, phase_i: n or
// null for the shared phase) into xv (n x 6) (hybrid.cu)
struct GCFullArgs {
    DevFields f;
    const double* y;
    const double* mu;
    const double* phase_i;
    int64_t n;
    double q, m, t, phase;
    double* xv;
};

// the work-rate columns of save_work, filled after a push over its saved
// states (slot-major: t[k n + i], u[(k W + c) n + i]) (gc_fp64.cu)
struct WorkFillArgs {
    DevFields f;
    const double* t_out;
    double* u_out;
    const int32_t* nsaved;
    int64_t n, nslots;
    int32_t W, c0, gc, pad;
    double q2m, m;           // full orbit
    double q, mu;            // guiding centre (scalars)
    const double* q_i;       // guiding centre, per particle (optional)
    const double* q2m_i;
    const double* mu_i;
};

// adaptive hybrid GC / full-orbit solve (hybrid.cu)
struct HybridArgs {
    DevFields f;
    DevTerm term;
    double t0, t1, q2m, m;
    double th_gc_fo, th_fo_gc, dtmin, dtmax, safety_fo, abstol, reltol;
    int64_t maxiters, check, ssi;
    int32_t adia_mode, save_adia, save_start, save_end, save_everystep, pad;
    int64_t n, nslots, aslots;
    const double* u0;      // n x 6
    double* t_out;         // nslots x n
    double* u_out;         // nslots x 6 x n
    int32_t* nsaved;
    int8_t* retcode;
    int64_t* nsteps;
    double* at_out;        // aslots x n: check times
    double* av_out;        // aslots x 2 x n: (adiabaticity, mode)
    int32_t* nadia;
    int32_t* status;
    uint64_t budget_ns;
};

// fields and work rates at given states (tp_eval_points)
struct PointsArgs {
    DevFields f;
    const double* u;   // n states, `stride` doubles each
    const double* t;   // n times
    int64_t n;
    int32_t stride, want, wout, kind;
    double q2m, m, q, mu;
    // optional per-point parameters (null: the scalar above)
    const double* q2m_i;
    const double* m_i;
    const double* q_i;
    const double* mu_i;
    double* out;       // n rows of wout doubles
};

// discrete adjoint of the fixed-step Boris map (adjoint.cu)
constexpr int kAdjCkWords = 12;  // checkpoint words per particle

struct AdjArgs {
    BorisArgs a;           // fields, q2m, t0, dt, FP32C wrap data, n, u0 (device, n x 6)
    int64_t nt;            // steps N
    int64_t K;             // steps per checkpoint segment
    int64_t S;             // checkpoints: max(1, ceil(N / K))
    double dt_final;       // dt of the final save's half update
    float* ckpt;           // [S][kAdjCkWords][n]: hi xyz, lo xyz, v.h xyz, v.l xyz
    double* u_final;       // n x 6
    const double* g_final; // n x 6: dL/d(x_N, v_N)
    double* g_u0;          // n x 6
    float* rec;            // [K][9][n]: per step of a segment, hi xyz, lo xyz, v xyz
    float4* g_eb;          // interleaved node-gradient table (2 float4 per node) or null
    float4* g_E;           // per-field node-gradient tables (1 float4 per node) or null
    float4* g_B;
    double* g_param;       // 6: analytic-field parameter gradients (E then B)
    int32_t G;             // node-gradient tables hold float32 values times 2^G
    int32_t pad;
    int32_t* need;         // device: largest node-contribution exponent of the pass
    float* lam;            // [8][n] cotangent state between segments (segmented path)
};

// field configuration of an adjoint run (FK_ANALYTIC / FK_EBGRID / FK_GENERIC)
int adjoint_field_config(const DevFields& f);
cudaError_t launch_adjoint_forward(const AdjArgs& a, int fk, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_adjoint_backward(const AdjArgs& a, int fk, const LaunchCfg& c, cudaStream_t s);
int64_t adjoint_record_words(int fk, int64_t K, int64_t n);
int64_t adjoint_state_words(int fk, int64_t K, int64_t n);
// E/B-grid segments of at most kFusedMaxK steps run the one-kernel backward
// (records in shared memory); longer ones the two kernels per segment
constexpr int64_t kFusedMaxK = 8;
bool adjoint_fused(int fk, int64_t K);
// sum of a node-gradient table (values times 2^-G) into out[0..2] (+=),
// entries k*stride + off
cudaError_t launch_table_sum(const float4* tab, int64_t nodes, int stride, int off, int G, double* out,
                             cudaStream_t s);
// node-gradient table -> user layout out[3*k + c] (float64, scaled back by 2^G)
cudaError_t launch_table_unpack(const float4* tab, int64_t nodes, int stride, int off, int G, double* out,
                                cudaStream_t s);

cudaError_t launch_boris_fp64(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_boris_fp32c(const BorisArgs& a, const LaunchCfg& c, cudaStream_t s);
// the FP32C run takes the warp-cooperative cubic-grid kernel (static schedule only)
bool fp32c_cubic_coop(const BorisArgs& a);
int occupancy_boris_fp64(const BorisArgs& a, int block);
int occupancy_boris_fp32c(const BorisArgs& a, int block);

cudaError_t launch_gc(const GCArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_gc_fp32(const GCArgs& a, const LaunchCfg& c, cudaStream_t s);
int occupancy_gc(const GCArgs& a, int block);
cudaError_t launch_gc_prepare(const GCPrepArgs& a, cudaStream_t s);
cudaError_t launch_eval_points(const PointsArgs& a, cudaStream_t s);
cudaError_t launch_fill_work(const WorkFillArgs& a, cudaStream_t s);
cudaError_t launch_hybrid(const HybridArgs& a, int block, cudaStream_t s);
cudaError_t launch_gc_to_full(const GCFullArgs& a, cudaStream_t s);
// Load the kernel a launch will use (cudaFuncGetAttributes), so that lazy
// module loading happens before a timed region instead of at the first launch
cudaError_t prime_boris_fp64(const BorisArgs& a);
cudaError_t prime_boris_fp32c(const BorisArgs& a);
cudaError_t prime_gc(const GCArgs& a);
cudaError_t prime_fill_work();
cudaError_t prime_hybrid(const HybridArgs& a);
// virtual detectors (detect.cu): mode 0 fluxes (tot: nsurf x 4 sums on the
// device), 1 crossings (counts on the host; *rows_d_out: device rows the
// caller frees with cudaFreeAsync), 2 first crossing (first: n x 6, device)
cudaError_t launch_detect(int mode, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                          int64_t n, const tp_surface* surf_d, int32_t nsurf, const double* weights,
                          double weight, double* tot, int64_t* counts_h, double** rows_d_out, double* first,
                          cudaStream_t s);

// context accessors for translation units outside runtime.cu
int ctx_device(const tp_ctx* ctx);
int ctx_fail(tp_ctx* ctx, int code, const std::string& msg);

// static-scratch packing (noalloc.cu)
int noalloc_scratch(int device, int64_t** out);
cudaError_t launch_noalloc_pack(int64_t* scratch, const double* t_in, const double* u_in,
                                const int32_t* nsaved, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, int64_t* total_out, cudaStream_t s);

// packing helpers (pack.cu)
// processing order of the particles by the Morton key of their initial cell
// on grid g (pack.cu); tmp = null sizes the scratch
cudaError_t cell_order(const double* u0, int64_t n, const DevField& g, void* tmp, size_t* tmp_bytes,
                       int32_t** perm, cudaStream_t s);
cudaError_t launch_pack_node_table(const void* src, int src_f64, int64_t nodes, void* dst,
                                   int dst_f64, int stride, int off, cudaStream_t s);
cudaError_t launch_pack_results(const double* t_in, const double* u_in, const int32_t* nsaved,
                                const int64_t* offsets, int64_t n, int64_t nslots, int width,
                                double* t_out, double* u_out, cudaStream_t s);

}  // namespace tpb
