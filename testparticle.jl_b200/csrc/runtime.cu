// runtime.cu -- host side of the C ABI (include/tp_abi.h).
//
// Owns the device, one stream per context, field uploads (grid data is laid
// out once as per-node 4-vectors; an E/B pair on one geometry is interleaved
// so each corner is one 32-byte sector), argument validation that mirrors the
// reference's ArgumentErrors, kernel launches, and result packing into the
// reference's per-trajectory layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "tp_launch.h"

namespace tpb {
cudaError_t scan_offsets(const int32_t* nsaved, int64_t n, int64_t nslots, int64_t* cnt,
                         int64_t* offsets, void* tmp, size_t* tmp_bytes, cudaStream_t s);
}

using namespace tpb;

struct tp_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // launch shapes chosen by tp_autotune, keyed by the kernel variant
    // (algorithm, precision, field configuration, termination): block, schedule
    struct Shape {
        int block, sched, ppt;
    };
    std::map<std::string, Shape> tuned;
    // pinned staging for host <-> device transfers of pageable buffers
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
    // tp_boris_run_host, created on first use and kept: pinned staging of
    // one chunk's slot-major results, the chunk counts' pinned mirror, the
    // copy stream and the two timing events
    void* chunk_pin = nullptr;
    size_t chunk_pin_bytes = 0;
    int32_t* done_pin = nullptr;
    int64_t done_cap = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t run_ev[2] = {nullptr, nullptr};
};

struct tp_field {
    tp_ctx* ctx = nullptr;
    uint64_t id = 0;
    tp_field_desc desc{};
    DevField dev{};
    int64_t nodes = 0;
    void* d_raw = nullptr;   // uploaded (3, nx, ny, nz) data
    void* d_tab = nullptr;   // per-node table in the data's precision
    void* d_tab32 = nullptr; // float per-node table (only for f64 data)
    // interleaved E/B table built on first use with a partner field
    uint64_t eb_partner = 0;
    void* d_eb = nullptr;
    void* d_eb32 = nullptr;
    // the same for two cubic periodic grids (k_cubic32c)
    uint64_t ebc_partner = 0;
    void* d_ebc32 = nullptr;
    void* d_axis[3] = {nullptr, nullptr, nullptr};  // node coordinates of non-uniform axes
    // SERIES: owned snapshot fields, their device descriptors and times
    std::vector<tp_field*> snaps;
    void* d_snaps = nullptr;
    void* d_times = nullptr;
    void* d_self = nullptr;  // the DevField in device memory (DevField::self)
};

// Results stay on the device until tp_result_copy moves them into the
// caller's buffers (one pass through pinned staging).
struct tp_result {
    tp_ctx* ctx = nullptr;
    int64_t n = 0;
    int32_t width = 0;
    int64_t total = 0;
    void* nsaved = nullptr;   // device, n x int32
    void* retcode = nullptr;  // device, n x int8
    void* nsteps = nullptr;   // device, n x int64
    void* t = nullptr;        // device, total x double (packed)
    void* u = nullptr;        // device, total x width x double (packed)
    double elapsed_ms = 0.0;
    cudaStream_t s = nullptr;  // the stream the buffers are ordered on
    ~tp_result() {
        for (void* q : {nsaved, retcode, nsteps, t, u})
            if (q) cudaFreeAsync(q, s);
    }
};

namespace {

std::mutex g_id_mu;
uint64_t g_next_id = 1;

int fail(tp_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(tp_ctx* ctx, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    cudaGetLastError();  // clear a sticky-free error
    return fail(ctx, TP_E_CUDA, m);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// RAII device buffer
// Stream that DBuf allocations of the calling thread are ordered on: the
// context stream of the entry point being served (AllocStream sets it).
thread_local cudaStream_t g_alloc_stream = nullptr;

struct AllocStream {
    cudaStream_t prev;
    explicit AllocStream(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
    ~AllocStream() { g_alloc_stream = prev; }
};

// Device buffer from the device's stream-ordered memory pool (the context
// raises the pool's release threshold, so freed blocks are reused by the
// next solve instead of going back to the driver).  Allocation and release
// are ordered on the context stream, after any work that still uses it.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t s = nullptr;
    ~DBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    cudaError_t alloc(size_t b) {
        bytes = b;
        s = g_alloc_stream;
        if (b == 0) return cudaSuccess;
        return cudaMallocAsync(&p, b, s);
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

// ---------------------------------------------------------------- host transfers
// Pageable host memory is copied through two pinned 64 MB staging buffers of
// the context: the DMA of one chunk overlaps the host-side copy of the
// previous one, and the host-side copy is split over threads, which also
// spreads the first-touch page faults of freshly allocated destinations.
constexpr size_t kPinChunk = (size_t)64 << 20;

void host_copy(void* dst, const void* src, size_t bytes) {
    const size_t per = (size_t)8 << 20;
    unsigned hw = std::thread::hardware_concurrency();
    int nt = (int)std::min<size_t>(std::max(1u, std::min(hw, 16u)), (bytes + per - 1) / per);
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t slice = (bytes + nt - 1) / nt;
    for (int k = 0; k < nt; ++k) {
        size_t a = (size_t)k * slice, b = std::min(bytes, a + slice);
        if (a >= b) break;
        th.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
    }
    for (auto& x : th) x.join();
}

cudaError_t ensure_pinned(tp_ctx* ctx) {
    for (int k = 0; k < 2; ++k) {
        if (!ctx->pin[k]) {
            cudaError_t e = cudaHostAlloc(&ctx->pin[k], kPinChunk, cudaHostAllocDefault);
            if (e != cudaSuccess) return e;
        }
        if (!ctx->pin_ev[k]) {
            cudaError_t e = cudaEventCreateWithFlags(&ctx->pin_ev[k], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

bool is_pageable(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return at.type == cudaMemoryTypeUnregistered;
}

// device -> host (dst may be pageable) on stream s; synchronous on return
cudaError_t copy_to_host_on(tp_ctx* ctx, cudaStream_t s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (bytes < ((size_t)4 << 20) || !is_pageable(dst)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    }
    cudaError_t e = ensure_pinned(ctx);
    if (e != cudaSuccess) return e;
    const size_t nch = (bytes + kPinChunk - 1) / kPinChunk;
    for (size_t k = 0; k <= nch; ++k) {
        if (k < nch) {
            size_t off = k * kPinChunk, len = std::min(kPinChunk, bytes - off);
            e = cudaMemcpyAsync(ctx->pin[k & 1], (const char*)src + off, len, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[k & 1], s);
            if (e != cudaSuccess) return e;
        }
        if (k > 0) {  // the previous chunk: wait for its DMA, then spread it out
            size_t j = k - 1, off = j * kPinChunk, len = std::min(kPinChunk, bytes - off);
            e = cudaEventSynchronize(ctx->pin_ev[j & 1]);
            if (e != cudaSuccess) return e;
            host_copy((char*)dst + off, ctx->pin[j & 1], len);
        }
    }
    return cudaSuccess;
}

cudaError_t copy_to_host(tp_ctx* ctx, void* dst, const void* src, size_t bytes) {
    return copy_to_host_on(ctx, ctx->stream, dst, src, bytes);
}

// host (possibly pageable) -> device on stream s; the call returns once the
// staging buffers are free again (the stream is synchronised when they were
// used)
cudaError_t copy_to_device_on(tp_ctx* ctx, cudaStream_t s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (bytes < ((size_t)4 << 20) || !is_pageable(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s);
    cudaError_t e = ensure_pinned(ctx);
    if (e != cudaSuccess) return e;
    const size_t nch = (bytes + kPinChunk - 1) / kPinChunk;
    for (size_t k = 0; k < nch; ++k) {
        size_t off = k * kPinChunk, len = std::min(kPinChunk, bytes - off);
        if (k >= 2) {  // the buffer's previous DMA must be done before refilling it
            e = cudaEventSynchronize(ctx->pin_ev[k & 1]);
            if (e != cudaSuccess) return e;
        }
        host_copy(ctx->pin[k & 1], (const char*)src + off, len);
        e = cudaMemcpyAsync((char*)dst + off, ctx->pin[k & 1], len, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_ev[k & 1], s);
        if (e != cudaSuccess) return e;
    }
    // the staging buffers are reused by the next transfer: finish this one
    return cudaStreamSynchronize(s);
}

cudaError_t copy_to_device(tp_ctx* ctx, void* dst, const void* src, size_t bytes) {
    return copy_to_device_on(ctx, ctx->stream, dst, src, bytes);
}

const double kEps = 2.220446049250313e-16;

int64_t jl_round_h(double x) { return (int64_t)std::nearbyint(x); }

int64_t nout_h(int64_t nt, int64_t ssi, bool ss, bool se, bool sev) {
    int64_t nout = 0;
    if (ss) nout += 1;
    if (sev) {
        int64_t steps = nt / ssi;
        bool last_is_step = (nt > 0) && (nt % ssi == 0);
        nout += steps;
        if (!se && last_is_step) nout -= 1;
        if (se && !last_is_step) nout += 1;
    } else if (se) {
        nout += 1;
    }
    return nout;
}

// Per-particle step counts of a fixed-step solve: the save slots needed (the
// largest nout over particles) and the first particle that breaks the
// reference's argument checks (boris.jl:349-356), in index order: dt below
// 10 eps (bad = 1) or |nt| above maxiters (bad = 2, nt reported).  Large
// ensembles are scanned by several host threads; the result is the serial
// loop's.
struct StepScan {
    int64_t nslots = 0;
    int64_t bad_index = -1;
    int bad = 0;
    int64_t bad_nt = 0;
};

StepScan scan_steps(const tp_run_desc* d, const double* dt_i, const double* tend_i, int64_t n) {
    const bool per = (dt_i || tend_i) && n > 0;
    const int64_t m = per ? n : 1;
    auto part = [&](int64_t a, int64_t b, StepScan& r) {
        for (int64_t i = a; i < b; ++i) {
            const double dt = (dt_i && n > 0) ? dt_i[i] : d->dt;
            const double t1 = (tend_i && n > 0) ? tend_i[i] : d->t1;
            if (std::fabs(dt) < 10.0 * kEps) {
                r.bad_index = i;
                r.bad = 1;
                return;
            }
            int64_t nt = jl_round_h((t1 - d->t0) / dt);
            if (nt < 0) nt = -nt;
            if (nt > d->maxiters) {
                r.bad_index = i;
                r.bad = 2;
                r.bad_nt = nt;
                return;
            }
            r.nslots = std::max(r.nslots, nout_h(nt, d->savestepinterval, d->save_start, d->save_end,
                                                 d->save_everystep));
        }
    };
    const int64_t per_thread = 1 << 16;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nth = (int)std::min<int64_t>(std::max(1u, std::min(hw, 32u)), (m + per_thread - 1) / per_thread);
    if (nth <= 1) {
        StepScan r;
        part(0, m, r);
        return r;
    }
    std::vector<StepScan> rs(nth);
    std::vector<std::thread> th;
    const int64_t slice = (m + nth - 1) / nth;
    for (int k = 0; k < nth; ++k)
        th.emplace_back(part, std::min(m, k * slice), std::min(m, (k + 1) * slice), std::ref(rs[k]));
    for (auto& t : th) t.join();
    StepScan r;
    for (const StepScan& q : rs) {  // slices in index order: the first bad one is the serial loop's
        if (q.bad) {
            r.bad_index = q.bad_index;
            r.bad = q.bad;
            r.bad_nt = q.bad_nt;
            return r;
        }
        r.nslots = std::max(r.nslots, q.nslots);
    }
    return r;
}

void fill_float_copies(DevField& d) {
    for (int a = 0; a < 3; ++a) {
        d.vf[a] = (float)d.v[a];
        d.ratef[a] = (float)d.rate[a];
        d.mf[a] = (float)d.m[a];
        d.cf[a] = (float)d.c[a];
        d.x0f[a] = (float)d.x0[a];
        d.dxf[a] = (float)(1.0 / d.inv_dx[a]);
        d.idxf[a] = (float)d.inv_dx[a];
    }
    for (int k = 0; k < 9; ++k) d.Jf[k] = (float)d.J[k];
    d.coeff = (float)d.coef;
    double mm = std::sqrt(d.m[0] * d.m[0] + d.m[1] * d.m[1] + d.m[2] * d.m[2]);
    for (int a = 0; a < 3; ++a) d.mhatf[a] = mm > 0 ? (float)(d.m[a] / mm) : 0.0f;
    d.Kf = (float)(d.coef * mm);
}

// Validation of a grid descriptor (the reference's build_interpolator
// errors, src/utility/interpolation.jl:126-311); empty when valid.
std::string check_grid_desc(const tp_field_desc* d) {
    if (d->bc < TP_BC_FILL_NAN || d->bc > TP_BC_PERIODIC_INCLUSIVE) return "unknown grid boundary condition";
    if (d->dtype != TP_DTYPE_F32 && d->dtype != TP_DTYPE_F64) return "grid dtype must be float32 or float64";
    if (!d->data) return "grid data pointer is null";
    if (d->order < TP_ORDER_LINEAR || d->order > TP_ORDER_CUBIC)
        return "Interpolation order is not supported. Supported orders are 0, 1, and 3.";
    if (d->geometry < TP_GRID_CARTESIAN || d->geometry > TP_GRID_SPHERICAL_SCALAR) return "unknown grid geometry";
    const bool sph = d->geometry != TP_GRID_CARTESIAN;
    if (d->ndim < 0 || d->ndim > 3 || (sph && d->ndim != 0 && d->ndim != 3)) return "grid ndim must be 1, 2 or 3";
    const int ndim = d->ndim == 0 ? 3 : d->ndim;
    if (ndim == 1 && (d->dir < 0 || d->dir > 2)) return "1-D grid dir must be 0, 1 or 2";
    int64_t nodes = 1;
    for (int k = 0; k < 3; ++k) {
        if (k >= ndim) {
            if (d->n[k] != 1) return "unused axes of a 1-D / 2-D grid must have n = 1";
            if (d->axis[k]) return "unused axes of a 1-D / 2-D grid take no node coordinates";
            continue;
        }
        if (d->n[k] < 2 || d->n[k] > (1 << 20)) return "grid needs 2 .. 2^20 nodes per axis";
        if (d->axis[k]) {
            const double* c = d->axis[k];
            for (int64_t i = 0; i < d->n[k]; ++i)
                if (!std::isfinite(c[i]) || (i > 0 && !(c[i] > c[i - 1])))
                    return "grid vectors must be finite and strictly increasing";
            if (d->order == TP_ORDER_CUBIC)
                return "RectilinearGrid (CartesianNonUniform) only supports order=1 (Linear) interpolation.";
            const bool periodic_axis =
                sph ? k == 2 : (d->bc == TP_BC_PERIODIC || d->bc == TP_BC_PERIODIC_INCLUSIVE);
            if (periodic_axis) return "periodic axes must be uniform";
        } else if (!(d->spacing[k] > 0.0) || !std::isfinite(d->spacing[k])) {
            return "grid spacing must be positive and finite";
        }
        nodes *= d->n[k];
    }
    if (nodes > ((int64_t)1 << 31) / 2) return "grid too large (more than 2^30 nodes)";
    if (sph) {
        // build_interpolator(StructuredGrid, ...) assertions (:270-280)
        double r0 = d->axis[0] ? d->axis[0][0] : d->origin[0];
        double t0 = d->axis[1] ? d->axis[1][0] : d->origin[1];
        double t1 = d->axis[1] ? d->axis[1][d->n[1] - 1] : d->origin[1] + (double)(d->n[1] - 1) * d->spacing[1];
        double p0 = d->origin[2], p1 = d->origin[2] + (double)(d->n[2] - 1) * d->spacing[2];
        const double pi = 3.141592653589793, eps = 1e-12;
        if (!(r0 >= 0.0)) return "r must be non-negative.";
        if (!(t0 >= -eps && t1 <= pi + eps)) return "theta must be within [0, pi].";
        if (!(p0 >= -eps && p1 <= 2.0 * pi + eps)) return "phi must be within [0, 2pi].";
    }
    return std::string();
}

bool same_geometry(const tp_field* a, const tp_field* b) {
    if (a->desc.kind != TP_FIELD_GRID || b->desc.kind != TP_FIELD_GRID) return false;
    if (a->dev.general || b->dev.general) return false;
    if (a->desc.bc != b->desc.bc || a->desc.dtype != b->desc.dtype) return false;
    for (int k = 0; k < 3; ++k) {
        if (a->desc.n[k] != b->desc.n[k]) return false;
        if (a->desc.origin[k] != b->desc.origin[k]) return false;
        if (a->desc.spacing[k] != b->desc.spacing[k]) return false;
    }
    return true;
}

// E and B both periodic (exclusive), uniform, Cartesian 3-D grids of order 3
// on one geometry with at least 4 nodes per axis: the interleaved float table
// of the warp-cooperative FP32C kernel
bool same_geometry_cubic(const tp_field* a, const tp_field* b) {
    for (const tp_field* f : {a, b}) {
        const tp_field_desc& d = f->desc;
        if (d.kind != TP_FIELD_GRID || d.order != TP_ORDER_CUBIC || d.geometry != TP_GRID_CARTESIAN) return false;
        if (!(d.ndim == 0 || d.ndim == 3) || d.bc != TP_BC_PERIODIC) return false;
        for (int k = 0; k < 3; ++k)
            if (d.axis[k] || d.n[k] < 4 || d.n[k] > (1 << 20)) return false;
    }
    for (int k = 0; k < 3; ++k) {
        if (a->desc.n[k] != b->desc.n[k]) return false;
        if (a->desc.origin[k] != b->desc.origin[k]) return false;
        if (a->desc.spacing[k] != b->desc.spacing[k]) return false;
    }
    return a->nodes <= ((int64_t)1 << 31) / 2;
}

DevTerm dev_term(const tp_term_desc& t) {
    DevTerm d{};
    d.flags = t.flags;
    d.rmin = t.rmin;
    d.rmax = t.rmax;
    for (int k = 0; k < 3; ++k) {
        d.lo[k] = t.lo[k];
        d.hi[k] = t.hi[k];
    }
    d.tmax = t.tmax;
    return d;
}

// Build DevFields for a run; interleaves two grids on one geometry.
int make_dev_fields(tp_ctx* ctx, const tp_field* E, tp_field* B, DevFields& F) {
    std::memset(&F, 0, sizeof(F));
    F.E = E->dev;
    F.B = B->dev;
    if (same_geometry(E, B)) {
        if (B->eb_partner != E->id) {
            if (B->d_eb) cudaFree(B->d_eb);
            if (B->d_eb32) cudaFree(B->d_eb32);
            B->d_eb = B->d_eb32 = nullptr;
            bool f64 = B->desc.dtype == TP_DTYPE_F64;
            size_t esz = f64 ? sizeof(double) : sizeof(float);
            cudaError_t e = cudaMalloc(&B->d_eb, (size_t)B->nodes * 8 * esz);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "interleaved field table");
            e = launch_pack_node_table(E->d_raw, f64, E->nodes, B->d_eb, f64, 2, 0, ctx->stream);
            if (e == cudaSuccess)
                e = launch_pack_node_table(B->d_raw, f64, B->nodes, B->d_eb, f64, 2, 1, ctx->stream);
            if (e == cudaSuccess && f64) {
                e = cudaMalloc(&B->d_eb32, (size_t)B->nodes * 8 * sizeof(float));
                if (e == cudaSuccess)
                    e = launch_pack_node_table(E->d_raw, 1, E->nodes, B->d_eb32, 0, 2, 0, ctx->stream);
                if (e == cudaSuccess)
                    e = launch_pack_node_table(B->d_raw, 1, B->nodes, B->d_eb32, 0, 2, 1, ctx->stream);
            }
            // the table is complete before any launch reads it: the entries
            // that take the caller's stream are not ordered after this one
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "interleaved field table");
            B->eb_partner = E->id;
        }
        F.eb = B->d_eb;
        F.eb_f64 = B->desc.dtype == TP_DTYPE_F64;
        F.eb32 = (const float4*)(B->d_eb32 ? B->d_eb32 : B->d_eb);
    } else if (same_geometry_cubic(E, B)) {
        if (B->ebc_partner != E->id) {
            if (B->d_ebc32) cudaFree(B->d_ebc32);
            B->d_ebc32 = nullptr;
            const int f64e = E->desc.dtype == TP_DTYPE_F64, f64b = B->desc.dtype == TP_DTYPE_F64;
            cudaError_t e = cudaMalloc(&B->d_ebc32, (size_t)B->nodes * 8 * sizeof(float));
            if (e == cudaSuccess) e = launch_pack_node_table(E->d_raw, f64e, E->nodes, B->d_ebc32, 0, 2, 0, ctx->stream);
            if (e == cudaSuccess) e = launch_pack_node_table(B->d_raw, f64b, B->nodes, B->d_ebc32, 0, 2, 1, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "interleaved cubic field table");
            B->ebc_partner = E->id;
        }
        F.ebc32 = (const float4*)B->d_ebc32;
    }
    return TP_OK;
}

// Periodic wrapping of FP32C positions: only on axes where every
// position-dependent field is a periodic grid with one period, and when no
// spatial termination predicate reads absolute positions.
void set_wrap(BorisArgs& a, const tp_field* E, const tp_field* B, const tp_term_desc& term) {
    for (int c = 0; c < 3; ++c) a.wrap[c] = 0;
    if (term.flags & (TP_TERM_SHELL | TP_TERM_BOX)) return;
    const tp_field* f[2] = {E, B};
    bool any_grid = false;
    for (int c = 0; c < 3; ++c) {
        bool ok = true;
        double L = 0, x0 = 0;
        bool have = false;
        for (const tp_field* g : f) {
            int k = g->desc.kind;
            if (k == TP_FIELD_ZERO || k == TP_FIELD_UNIFORM) continue;
            if (k == TP_FIELD_AFFINE) {
                // translation-invariant only if it does not depend on this axis
                for (int r = 0; r < 3; ++r)
                    if (g->desc.jac[3 * r + c] != 0.0) ok = false;
                continue;
            }
            // trilinear grids, and cubic ones on uniform Cartesian 3-D axes:
            // exclusive-periodic with period n dx on every axis
            const bool cubic_uniform = g->desc.order == TP_ORDER_CUBIC && g->desc.geometry == TP_GRID_CARTESIAN &&
                                       (g->desc.ndim == 0 || g->desc.ndim == 3) && !g->desc.axis[0] &&
                                       !g->desc.axis[1] && !g->desc.axis[2];
            if (k != TP_FIELD_GRID || g->desc.bc != TP_BC_PERIODIC || (g->dev.general && !cubic_uniform)) {
                ok = false;
                continue;
            }
            double Lg = (double)g->desc.n[c] * g->desc.spacing[c];
            if (have && (Lg != L || g->desc.origin[c] != x0)) ok = false;
            L = Lg;
            x0 = g->desc.origin[c];
            have = true;
            any_grid = true;
        }
        if (ok && have) {
            a.wrap[c] = 1;
            a.wrapL[c] = L;
            a.wrap0[c] = x0;
        }
    }
    (void)any_grid;
}

int check_boris_desc(tp_ctx* ctx, const tp_run_desc* d) {
    if (!d) return fail(ctx, TP_E_ARG, "null run descriptor");
    if (d->alg < TP_ALG_BORIS || d->alg > TP_ALG_ADAPTIVE_MULTISTEP)
        return fail(ctx, TP_E_UNSUPPORTED, "unknown algorithm");
    bool multi = d->alg == TP_ALG_MULTISTEP || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (multi && d->order != 2 && d->order != 4 && d->order != 6)
        return fail(ctx, TP_E_ARG, "Multistep Boris order N must be 2, 4, or 6.");
    if (multi && d->nsub < 1) return fail(ctx, TP_E_ARG, "Multistep Boris subcycles n must be >= 1");
    if (d->savestepinterval < 1) return fail(ctx, TP_E_ARG, "savestepinterval must be >= 1");
    if (d->precision != TP_PREC_FP64 && d->precision != TP_PREC_FP32C)
        return fail(ctx, TP_E_UNSUPPORTED, "unknown precision");
    if (d->block < 0 || d->block > 384 || (d->block % 32) != 0)
        return fail(ctx, TP_E_ARG, "block must be 0 or a multiple of 32 up to 384");
    if (d->schedule < TP_SCHED_AUTO || d->schedule > TP_SCHED_QUEUE)
        return fail(ctx, TP_E_ARG, "unknown schedule");
    return TP_OK;
}

// Static schedule: one thread per particle.  Queue schedule: a persistent
// grid of (SMs x resident blocks) pulling particles from a device counter.
int pick_launch(tp_ctx* ctx, int64_t n, int block_req, bool queue, int occ_blocks, LaunchCfg& cfg) {
    int block = block_req > 0 ? block_req : 128;
    int64_t need = (n + block - 1) / block;
    if (need < 1) need = 1;
    if (need > 0x7fffffff) return fail(ctx, TP_E_ARG, "too many particles for one launch");
    cfg.block = block;
    if (!queue) {
        cfg.grid = (int)need;
        return TP_OK;
    }
    int64_t resident = (int64_t)ctx->sms * std::max(occ_blocks, 1);
    cfg.grid = (int)std::min<int64_t>(need, resident);
    return TP_OK;
}

}  // namespace

// ============================================================== C ABI
extern "C" {

int tp_abi_version(void) { return TP_ABI_VERSION; }

int tp_ctx_create(int device, tp_ctx** out) {
    if (!out) return TP_E_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return TP_E_CUDA;
    }
    if (device < 0 || device >= ndev) return TP_E_ARG;
    DeviceGuard g(device);
    tp_ctx* c = new tp_ctx();
    c->device = device;
    e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // keep freed pool memory in this process for the next solve
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    if (e != cudaSuccess) {
        delete c;
        cudaGetLastError();
        return TP_E_CUDA;
    }
    *out = c;
    return TP_OK;
}

void tp_ctx_destroy(tp_ctx* ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int k = 0; k < 2; ++k) {
        if (ctx->pin[k]) cudaFreeHost(ctx->pin[k]);
        if (ctx->pin_ev[k]) cudaEventDestroy(ctx->pin_ev[k]);
    }
    if (ctx->chunk_pin) cudaFreeHost(ctx->chunk_pin);
    if (ctx->done_pin) cudaFreeHost(ctx->done_pin);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    for (cudaEvent_t ev : ctx->run_ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* tp_last_error(const tp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tp_field_create(tp_ctx* ctx, const tp_field_desc* d, tp_field** out) {
    if (!ctx || !d || !out) return fail(ctx, TP_E_ARG, "null argument");
    *out = nullptr;
    DeviceGuard g(ctx->device);
    tp_field* f = new tp_field();
    f->ctx = ctx;
    {
        std::lock_guard<std::mutex> lk(g_id_mu);
        f->id = g_next_id++;
    }
    f->desc = *d;
    f->desc.data = nullptr;
    DevField& dv = f->dev;
    std::memset(&dv, 0, sizeof(dv));
    dv.kind = d->kind;
    dv.bc = d->bc;
    for (int k = 0; k < 3; ++k) {
        dv.v[k] = d->value[k];
        dv.rate[k] = d->rate[k];
        dv.m[k] = d->moment[k];
        dv.c[k] = d->center[k];
    }
    for (int k = 0; k < 9; ++k) dv.J[k] = d->jac[k];
    dv.coef = d->coef;
    switch (d->kind) {
        case TP_FIELD_ZERO:
        case TP_FIELD_UNIFORM:
        case TP_FIELD_AFFINE:
        case TP_FIELD_DIPOLE:
            break;
        case TP_FIELD_QUADRATIC:
            for (int k = 0; k < 27; ++k) dv.Q[k] = d->quad[k];
            break;
        case TP_FIELD_SERIES: {
            // LazyTimeInterpolator: every snapshot uploaded once, resident
            const int64_t ns = d->nseries;
            if (ns < 1 || ns > (1 << 20) || !d->series || !d->series_times) {
                delete f;
                return fail(ctx, TP_E_ARG, "a series needs 1 .. 2^20 snapshots with times");
            }
            for (int64_t k = 0; k < ns; ++k) {
                if (!std::isfinite(d->series_times[k]) || (k > 0 && d->series_times[k] < d->series_times[k - 1])) {
                    delete f;
                    return fail(ctx, TP_E_ARG, "series times must be finite and sorted");
                }
                if (d->series[k].kind == TP_FIELD_SERIES) {
                    delete f;
                    return fail(ctx, TP_E_ARG, "a series snapshot cannot be a series");
                }
            }
            f->desc.series = nullptr;
            f->desc.series_times = nullptr;
            std::vector<DevField> devs((size_t)ns);
            for (int64_t k = 0; k < ns; ++k) {
                tp_field* c = nullptr;
                int st = tp_field_create(ctx, &d->series[k], &c);
                if (st != TP_OK) {
                    tp_field_destroy(f);
                    return st;
                }
                f->snaps.push_back(c);
                devs[(size_t)k] = c->dev;
            }
            cudaError_t e = cudaMalloc(&f->d_snaps, (size_t)ns * sizeof(DevField));
            if (e == cudaSuccess) e = cudaMalloc(&f->d_times, (size_t)ns * sizeof(double));
            if (e == cudaSuccess)
                e = cudaMemcpy(f->d_snaps, devs.data(), (size_t)ns * sizeof(DevField), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMemcpy(f->d_times, d->series_times, (size_t)ns * sizeof(double), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                int r = cuda_fail(ctx, e, "series upload");
                tp_field_destroy(f);
                return r;
            }
            dv.snaps = (const DevField*)f->d_snaps;
            dv.ts = (const double*)f->d_times;
            dv.nts = (int32_t)ns;
            break;
        }
        case TP_FIELD_GRID: {
            std::string why = check_grid_desc(d);
            if (!why.empty()) {
                delete f;
                return fail(ctx, TP_E_ARG, why);
            }
            const bool sph = d->geometry != TP_GRID_CARTESIAN;
            const int ndim = sph ? 3 : (d->ndim == 0 ? 3 : d->ndim);
            dv.order = d->order;
            dv.geom = d->geometry;
            dv.ndim = ndim;
            dv.dir = d->dir;
            for (int k = 0; k < 3; ++k) dv.abc[k] = d->bc;
            if (sph) {
                // SphericalFieldInterpolator: r and theta fill NaN, phi periodic
                // (interpolation.jl:150-164)
                dv.abc[0] = TP_BC_FILL_NAN;
                dv.abc[1] = TP_BC_FILL_NAN;
                dv.abc[2] = TP_BC_PERIODIC_INCLUSIVE;
            }
            bool general = d->order != TP_ORDER_LINEAR || d->geometry != TP_GRID_CARTESIAN || ndim != 3 ||
                           d->bc == TP_BC_PERIODIC_INCLUSIVE;
            int64_t nodes = 1;
            for (int k = 0; k < 3; ++k) {
                nodes *= d->n[k];
                dv.n[k] = (int32_t)d->n[k];
                if (d->axis[k]) {
                    general = true;
                    dv.x0[k] = d->axis[k][0];
                    dv.inv_dx[k] = 1.0;
                    dv.L[k] = d->axis[k][d->n[k] - 1] - d->axis[k][0];
                } else {
                    double sp = d->n[k] == 1 ? 1.0 : d->spacing[k];
                    dv.x0[k] = d->origin[k];
                    dv.inv_dx[k] = 1.0 / sp;
                    dv.L[k] = (double)d->n[k] * sp;
                }
            }
            dv.general = general ? 1 : 0;
            for (int k = 0; k < 3; ++k) {
                if (!d->axis[k]) continue;
                cudaError_t e = cudaMalloc(&f->d_axis[k], (size_t)d->n[k] * sizeof(double));
                if (e == cudaSuccess)
                    e = cudaMemcpy(f->d_axis[k], d->axis[k], (size_t)d->n[k] * sizeof(double),
                                   cudaMemcpyDefault);
                if (e != cudaSuccess) {
                    int r = cuda_fail(ctx, e, "grid axis upload");
                    tp_field_destroy(f);
                    return r;
                }
                dv.ax[k] = (const double*)f->d_axis[k];
            }
            f->nodes = nodes;
            bool f64 = d->dtype == TP_DTYPE_F64;
            size_t esz = f64 ? sizeof(double) : sizeof(float);
            cudaError_t e = cudaMalloc(&f->d_raw, (size_t)nodes * 3 * esz);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(f->d_raw, d->data, (size_t)nodes * 3 * esz, cudaMemcpyDefault,
                                    ctx->stream);
            if (e == cudaSuccess) e = cudaMalloc(&f->d_tab, (size_t)nodes * 4 * esz);
            if (e == cudaSuccess)
                e = launch_pack_node_table(f->d_raw, f64, nodes, f->d_tab, f64, 1, 0, ctx->stream);
            if (e == cudaSuccess && f64) {
                e = cudaMalloc(&f->d_tab32, (size_t)nodes * 4 * sizeof(float));
                if (e == cudaSuccess)
                    e = launch_pack_node_table(f->d_raw, 1, nodes, f->d_tab32, 0, 1, 0, ctx->stream);
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) {
                int r = cuda_fail(ctx, e, "grid upload");
                tp_field_destroy(f);
                return r;
            }
            dv.f64 = f64;
            dv.tab = f->d_tab;
            dv.tab32 = (const float4*)(f64 ? f->d_tab32 : f->d_tab);
            break;
        }
        default:
            delete f;
            return fail(ctx, TP_E_UNSUPPORTED, "field kind not supported by the B200 library");
    }
    fill_float_copies(dv);
    {
        cudaError_t e = cudaMalloc(&f->d_self, sizeof(DevField));
        if (e == cudaSuccess) {
            dv.self = (const DevField*)f->d_self;
            e = cudaMemcpy(f->d_self, &dv, sizeof(DevField), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            int r = cuda_fail(ctx, e, "field descriptor upload");
            tp_field_destroy(f);
            return r;
        }
    }
    *out = f;
    return TP_OK;
}

int tp_field_update(tp_field* f, const void* data) {
    if (!f) return TP_E_ARG;
    tp_ctx* ctx = f->ctx;
    if (f->desc.kind != TP_FIELD_GRID) return fail(ctx, TP_E_ARG, "tp_field_update needs a grid field");
    if (!data) return fail(ctx, TP_E_ARG, "grid data pointer is null");
    DeviceGuard g(ctx->device);
    bool f64 = f->desc.dtype == TP_DTYPE_F64;
    size_t esz = f64 ? sizeof(double) : sizeof(float);
    cudaError_t e = cudaMemcpyAsync(f->d_raw, data, (size_t)f->nodes * 3 * esz, cudaMemcpyDefault, ctx->stream);
    if (e == cudaSuccess) e = launch_pack_node_table(f->d_raw, f64, f->nodes, f->d_tab, f64, 1, 0, ctx->stream);
    if (e == cudaSuccess && f64)
        e = launch_pack_node_table(f->d_raw, 1, f->nodes, f->d_tab32, 0, 1, 0, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "grid update");
    // new identity: interleaved tables built with the old values are rebuilt
    {
        std::lock_guard<std::mutex> lk(g_id_mu);
        f->id = g_next_id++;
    }
    f->eb_partner = 0;
    return TP_OK;
}

void tp_field_destroy(tp_field* f) {
    if (!f) return;
    DeviceGuard g(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    for (void* p : {f->d_raw, f->d_tab, f->d_tab32, f->d_eb, f->d_eb32, f->d_ebc32, f->d_axis[0], f->d_axis[1], f->d_axis[2],
                    f->d_snaps, f->d_times, f->d_self})
        if (p) cudaFree(p);
    for (tp_field* c : f->snaps) tp_field_destroy(c);
    delete f;
}

int tp_boris_slots(const tp_run_desc* d, const double* dt_i, const double* tend_i, int64_t n,
                   int64_t* nslots) {
    if (!d || !nslots || n < 0) return TP_E_ARG;
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (d->savestepinterval < 1) return TP_E_ARG;
    if (adaptive) {
        if (d->step_cap <= 0) {
            *nslots = -1;  // unknown: the run grows its buffers
            return TP_OK;
        }
        int64_t s = (d->save_start ? 1 : 0) + 1;
        if (d->save_everystep) s += d->step_cap / d->savestepinterval + 1;
        *nslots = s;
        return TP_OK;
    }
    const StepScan sc = scan_steps(d, dt_i, tend_i, n);
    if (sc.bad) return TP_E_ARG;
    *nslots = sc.nslots;
    return TP_OK;
}

}  // extern "C"

namespace {

// Fill the launch block of a full-orbit run (device pointers set by caller).
int prepare_boris_args(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, tp_field* B,
                       BorisArgs& a) {
    std::memset(&a, 0, sizeof(a));
    int st = make_dev_fields(ctx, E, B, a.f);
    if (st != TP_OK) return st;
    a.term = dev_term(d->term);
    a.alg = d->alg;
    a.order = d->order;
    a.nsub = d->nsub;
    a.save_fields = d->save_fields;
    a.save_work = d->save_work;
    a.save_start = d->save_start;
    a.save_end = d->save_end;
    a.save_everystep = d->save_everystep;
    a.safety = d->safety;
    a.t0 = d->t0;
    a.t1 = d->t1;
    a.dt = d->dt;
    a.q2m = d->q2m;
    a.m = d->m;
    a.ssi = d->savestepinterval;
    a.maxiters = d->maxiters;
    a.step_cap = d->step_cap;
    double budget = d->budget_s > 0 ? d->budget_s : 600.0;
    a.budget_ns = (uint64_t)(budget * 1e9);
    if (d->precision == TP_PREC_FP32C) set_wrap(a, E, B, d->term);
    return TP_OK;
}

// key of the kernel variant a run selects (what tp_autotune tunes)
std::string tune_key(const tp_run_desc* d, const BorisArgs& a) {
    return std::to_string(d->alg) + ":" + std::to_string(d->precision) + ":" +
           std::to_string(field_config_of(a.f)) + ":" + std::to_string(d->term.flags != 0);
}

// Effective block size, schedule and particles per thread of a run: the
// descriptor's, else the tuned ones, else 128 threads, one particle per
// thread and the queue whenever lifetimes can be uneven (adaptive steps or a
// termination predicate).
void resolve_launch(tp_ctx* ctx, const tp_run_desc* d, const BorisArgs& a, int& block, bool& queue, int& ppt) {
    block = d->block;
    int sched = d->schedule;
    ppt = d->particles_per_thread;
    if (block == 0 || sched == TP_SCHED_AUTO || ppt == 0) {
        auto it = ctx->tuned.find(tune_key(d, a));
        if (it != ctx->tuned.end()) {
            if (block == 0) block = it->second.block;
            if (sched == TP_SCHED_AUTO) sched = it->second.sched;
            if (ppt == 0) ppt = it->second.ppt;
        }
    }
    if (block == 0) block = 128;
    if (ppt == 0) ppt = 1;
    if (sched == TP_SCHED_AUTO)
        sched = (d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP || d->term.flags != 0)
                    ? TP_SCHED_QUEUE
                    : TP_SCHED_STATIC;
    queue = sched == TP_SCHED_QUEUE;
}

bool use_queue(tp_ctx* ctx, const tp_run_desc* d, const BorisArgs& a) {
    int block, ppt;
    bool q;
    resolve_launch(ctx, d, a, block, q, ppt);
    return q;
}

// two particles per thread exist for the fixed-step analytic-field kernels
bool ppt2_available(const tp_run_desc* d, const BorisArgs& a) {
    return (d->alg == TP_ALG_BORIS || d->alg == TP_ALG_MULTISTEP) && field_config_of(a.f) == FK_ANALYTIC;
}

// launch shape of a run (host-only work: safe before a stream capture)
int plan_boris_launch(tp_ctx* ctx, const tp_run_desc* d, BorisArgs& a, LaunchCfg& cfg) {
    int block, ppt;
    bool q;
    resolve_launch(ctx, d, a, block, q, ppt);
    if (ppt != 1 && ppt != 2) return fail(ctx, TP_E_ARG, "particles_per_thread must be 0, 1 or 2");
    if (ppt == 2 && !ppt2_available(d, a)) ppt = 1;
    if (d->precision == TP_PREC_FP32C && fp32c_cubic_coop(a)) {
        q = false;  // the warp-cooperative kernel walks one particle per lane, static
        if (block > 128) block = 128;
    }
    if (block > TPB_MAXT(field_config_of(a.f)) / ppt)
        return fail(ctx, TP_E_ARG, "block exceeds the kernel's limit for this field configuration");
    a.use_queue = q;
    a.ppt = ppt;
    cudaError_t e = d->precision == TP_PREC_FP32C ? prime_boris_fp32c(a) : prime_boris_fp64(a);
    if (e == cudaSuccess && a.save_work) e = prime_fill_work();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel load");
    int occ = 0;
    if (q) occ = d->precision == TP_PREC_FP32C ? occupancy_boris_fp32c(a, block) : occupancy_boris_fp64(a, block);
    return pick_launch(ctx, (a.n + ppt - 1) / ppt, block, q, occ, cfg);
}

// the stream work of a run: queue reset and the push kernel
int issue_boris_launch(tp_ctx* ctx, const tp_run_desc* d, BorisArgs& a, const LaunchCfg& cfg, cudaStream_t s,
                       unsigned long long* d_queue) {
    a.queue = d_queue;
    if (a.use_queue) {
        cudaError_t e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "queue reset");
    }
    cudaError_t e = d->precision == TP_PREC_FP32C ? launch_boris_fp32c(a, cfg, s)
                                                  : launch_boris_fp64(a, cfg, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "push kernel launch");
    if (a.save_work && a.nslots > 0) {
        WorkFillArgs w;
        std::memset(&w, 0, sizeof(w));
        w.f = a.f;
        w.t_out = a.t_out;
        w.u_out = a.u_out;
        w.nsaved = a.nsaved;
        w.n = a.n;
        w.nslots = a.nslots;
        w.c0 = a.save_fields ? 12 : 6;
        w.W = w.c0 + 4;
        w.q2m = a.q2m;
        w.m = a.m;
        e = launch_fill_work(w, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "work-rate pass");
    }
    return TP_OK;
}

// Processing order of a solve in gridded fields (Cartesian geometry, n >=
// 65536): the particles sorted by the Morton key of their initial cell, so
// that the lanes of a warp gather neighbouring nodes (one radix sort of n
// keys, in the solve's device time).  Results do not depend on the order.
// The scratch comes from the pool on stream s; the caller releases *buf
// there after the push.
int order_particles(tp_ctx* ctx, BorisArgs& a, cudaStream_t s, void** buf) {
    *buf = nullptr;
    a.perm = nullptr;
    const DevField* g = nullptr;
    if (a.f.B.kind == TP_FIELD_GRID && a.f.B.geom == TP_GRID_CARTESIAN) g = &a.f.B;
    else if (a.f.E.kind == TP_FIELD_GRID && a.f.E.geom == TP_GRID_CARTESIAN) g = &a.f.E;
    if (!g || a.n < 65536 || a.n > 0x7fffffffLL) return TP_OK;
    size_t bytes = 0;
    cudaError_t e = cell_order(a.u0, a.n, *g, nullptr, &bytes, nullptr, s);
    if (e == cudaSuccess) e = cudaMallocAsync(buf, bytes, s);
    int32_t* perm = nullptr;
    if (e == cudaSuccess) e = cell_order(a.u0, a.n, *g, *buf, &bytes, &perm, s);
    if (e != cudaSuccess) {
        if (*buf) cudaFreeAsync(*buf, s);
        *buf = nullptr;
        return cuda_fail(ctx, e, "particle cell ordering");
    }
    a.perm = perm;
    return TP_OK;
}

int launch_boris(tp_ctx* ctx, const tp_run_desc* d, BorisArgs& a, cudaStream_t s,
                 unsigned long long* d_queue) {
    LaunchCfg cfg;
    int st = plan_boris_launch(ctx, d, a, cfg);
    if (st != TP_OK) return st;
    return issue_boris_launch(ctx, d, a, cfg, s, d_queue);
}

int status_to_error(tp_ctx* ctx, int32_t status) {
    switch (status) {
        case 0:
            return TP_OK;
        case TP_E_ARG:
            return fail(ctx, TP_E_ARG, "invalid per-particle dt / tspan (|dt| < 10 eps or nt > maxiters)");
        case TP_E_TIMEOUT:
            return fail(ctx, TP_E_TIMEOUT, "device loop exceeded its wall-clock budget");
        case TP_E_OVERFLOW:
            return fail(ctx, TP_E_OVERFLOW, "a trajectory produced more saves than slots");
        default:
            return fail(ctx, TP_E_CUDA, "kernel reported status " + std::to_string(status));
    }
}

// Copy slot-major device results into a packed host tp_result.
// Pack slot-major device results into the per-trajectory layout, on the
// device, into buffers the result owns; the per-particle arrays are moved
// into the result.
int pack_results(tp_ctx* ctx, int64_t n, int64_t nslots, int W, const DBuf& t_d, const DBuf& u_d, DBuf& ns_d,
                 DBuf& rc_d, DBuf& nst_d, tp_result* r) {
    cudaStream_t s = ctx->stream;
    r->ctx = ctx;
    r->s = s;
    r->n = n;
    r->width = W;
    if (n == 0) return TP_OK;
    DBuf cnt, off, tmp;
    size_t tmp_bytes = 0;
    cudaError_t e = cnt.alloc((size_t)(n + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = off.alloc((size_t)(n + 1) * sizeof(int64_t));
    if (e == cudaSuccess)
        e = scan_offsets(ns_d.as<int32_t>(), n, nslots, cnt.as<int64_t>(), off.as<int64_t>(), nullptr,
                         &tmp_bytes, s);
    if (e == cudaSuccess) e = tmp.alloc(tmp_bytes);
    if (e == cudaSuccess)
        e = scan_offsets(ns_d.as<int32_t>(), n, nslots, cnt.as<int64_t>(), off.as<int64_t>(), tmp.p,
                         &tmp_bytes, s);
    int64_t total = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&total, off.as<int64_t>() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "result offsets");
    r->total = total;
    e = cudaMallocAsync(&r->t, (size_t)std::max<int64_t>(total, 1) * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&r->u, (size_t)std::max<int64_t>(total, 1) * W * sizeof(double), s);
    if (e == cudaSuccess)
        e = launch_pack_results(t_d.as<double>(), u_d.as<double>(), ns_d.as<int32_t>(), off.as<int64_t>(),
                                n, nslots, W, (double*)r->t, (double*)r->u, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "result packing");
    r->nsaved = ns_d.p;
    r->retcode = rc_d.p;
    r->nsteps = nst_d.p;
    ns_d.p = rc_d.p = nst_d.p = nullptr;
    return TP_OK;
}

}  // namespace

extern "C" {

int tp_boris_run_device(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, const tp_field* B,
                        const double* u0, const double* dt_i, const double* tend_i, int64_t n,
                        int64_t nslots, double* t_out, double* u_out, int32_t* nsaved,
                        int8_t* retcode, int64_t* nsteps, int32_t* status, void* stream) {
    if (!ctx) return TP_E_ARG;
    int st = check_boris_desc(ctx, d);
    if (st != TP_OK) return st;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (n < 0 || nslots < 0) return fail(ctx, TP_E_ARG, "negative size");
    if (n == 0) return TP_OK;
    if (!u0 || !nsaved || !retcode || !nsteps || !status || (nslots > 0 && (!t_out || !u_out)))
        return fail(ctx, TP_E_ARG, "null device buffer");
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (!adaptive && !dt_i && std::fabs(d->dt) < 10.0 * kEps)
        return fail(ctx, TP_E_ARG, "time step dt is too small, violating min_dt = 10 * eps(typeof(dt))");
    DeviceGuard g(ctx->device);
    BorisArgs a;
    st = prepare_boris_args(ctx, d, E, const_cast<tp_field*>(B), a);
    if (st != TP_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    // the interleaved table (if any) was built on the context stream
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "field table");
    a.n = n;
    a.nslots = nslots;
    a.u0 = u0;
    a.dt_i = dt_i;
    a.tend_i = tend_i;
    a.t_out = t_out;
    a.u_out = u_out;
    a.nsaved = nsaved;
    a.retcode = retcode;
    a.nsteps = nsteps;
    a.status = status;
    unsigned long long* q = nullptr;
    if (use_queue(ctx, d, a)) {
        e = cudaMallocAsync((void**)&q, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "queue counter");
    }
    void* obuf = nullptr;
    st = order_particles(ctx, a, s, &obuf);
    if (st == TP_OK) st = launch_boris(ctx, d, a, s, q);
    if (obuf) cudaFreeAsync(obuf, s);
    if (q) cudaFreeAsync(q, s);
    return st;
}

int tp_autotune(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, const tp_field* B, const double* u0,
                int64_t n, int64_t max_steps, tp_tune_result* out) {
    if (!ctx || !out) return TP_E_ARG;
    int st = check_boris_desc(ctx, d);
    if (st != TP_OK) return st;
    if (!E || !B || !u0 || n <= 0) return fail(ctx, TP_E_ARG, "autotune needs fields and initial states");
    if (max_steps < 1) return fail(ctx, TP_E_ARG, "max_steps must be >= 1");
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (!adaptive && std::fabs(d->dt) < 10.0 * kEps) return fail(ctx, TP_E_ARG, "dt too small");
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    // the sample: first particles, span cut to max_steps
    tp_run_desc ds = *d;
    if (adaptive) {
        ds.step_cap = (ds.step_cap > 0 && ds.step_cap < max_steps) ? ds.step_cap : max_steps;
    } else {
        int64_t nt = jl_round_h((d->t1 - d->t0) / d->dt);
        if (nt < 0) nt = -nt;
        if (nt > max_steps) ds.t1 = d->t0 + (double)max_steps * d->dt;
    }
    const int64_t ns = std::min<int64_t>(n, 131072);
    int64_t nslots = 0;
    st = tp_boris_slots(&ds, nullptr, nullptr, ns, &nslots);
    if (st != TP_OK) return fail(ctx, st, "autotune sample sizing");
    const int W = 6 + (ds.save_fields ? 6 : 0) + (ds.save_work ? 4 : 0);
    DBuf u0_d, t_d, u_d, ns_d, rc_d, nst_d, st_d, q_d;
    cudaError_t e = u0_d.alloc((size_t)ns * 6 * sizeof(double));
    if (e == cudaSuccess) e = t_d.alloc((size_t)std::max<int64_t>(nslots, 1) * ns * sizeof(double));
    if (e == cudaSuccess) e = u_d.alloc((size_t)std::max<int64_t>(nslots, 1) * W * ns * sizeof(double));
    if (e == cudaSuccess) e = ns_d.alloc((size_t)ns * sizeof(int32_t));
    if (e == cudaSuccess) e = rc_d.alloc((size_t)ns * sizeof(int8_t));
    if (e == cudaSuccess) e = nst_d.alloc((size_t)ns * sizeof(int64_t));
    if (e == cudaSuccess) e = st_d.alloc(sizeof(int32_t));
    if (e == cudaSuccess) e = q_d.alloc(sizeof(unsigned long long));
    if (e == cudaSuccess) e = copy_to_device(ctx, u0_d.p, u0, (size_t)ns * 6 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(st_d.p, 0, sizeof(int32_t), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, std::string("autotune buffers: ") + cudaGetErrorString(e));
    BorisArgs a;
    st = prepare_boris_args(ctx, &ds, E, const_cast<tp_field*>(B), a);
    if (st != TP_OK) return st;
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "field table");
    a.n = ns;
    a.nslots = nslots;
    a.u0 = u0_d.as<double>();
    a.t_out = t_d.as<double>();
    a.u_out = u_d.as<double>();
    a.nsaved = ns_d.as<int32_t>();
    a.retcode = rc_d.as<int8_t>();
    a.nsteps = nst_d.as<int64_t>();
    a.status = st_d.as<int32_t>();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto time_shape = [&](int block, int sched, int ppt, double& ms) -> int {
        tp_run_desc dc = ds;
        dc.block = block;
        dc.schedule = sched;
        dc.particles_per_thread = ppt;
        float best = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {  // the first run warms up
            BorisArgs ac = a;
            cudaEventRecord(e0, ctx->stream);
            int r = launch_boris(ctx, &dc, ac, ctx->stream, q_d.as<unsigned long long>());
            if (r != TP_OK) return r;
            cudaEventRecord(e1, ctx->stream);
            cudaError_t ee = cudaEventSynchronize(e1);
            if (ee != cudaSuccess) return cuda_fail(ctx, ee, "autotune run");
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) best = std::min(best, t);
        }
        ms = best;
        return TP_OK;
    };
    const std::string key = tune_key(&ds, a);
    const int maxt = TPB_MAXT(field_config_of(a.f));
    const int blocks[] = {64, 96, 128, 192, 256, 384};
    int best_b = 128, best_s = TP_SCHED_STATIC, best_p = 1, cands = 0;
    double best_ms = 1e300, def_ms = 0.0;
    // the default shape, with any earlier tuning of this variant set aside
    auto saved = ctx->tuned.find(key);
    bool had = saved != ctx->tuned.end();
    tp_ctx::Shape old = had ? saved->second : tp_ctx::Shape{0, 0, 0};
    if (had) ctx->tuned.erase(key);
    st = time_shape(0, TP_SCHED_AUTO, 1, def_ms);
    // With uneven lifetimes (adaptive steps, termination) a cut sample has
    // even ones and would favour the static schedule: only the queue is
    // timed there.
    const bool uneven = adaptive || ds.term.flags != 0;
    const int max_ppt = ppt2_available(&ds, a) ? 2 : 1;
    for (int pp = 1; pp <= max_ppt; ++pp) {
        for (int b : blocks) {
            if (st != TP_OK) break;
            if (b > maxt / pp) continue;
            for (int sc : {TP_SCHED_STATIC, TP_SCHED_QUEUE}) {
                if (uneven && sc == TP_SCHED_STATIC) continue;
                double ms = 0.0;
                st = time_shape(b, sc, pp, ms);
                if (st != TP_OK) break;
                ++cands;
                if (ms < best_ms) {
                    best_ms = ms;
                    best_b = b;
                    best_s = sc;
                    best_p = pp;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != TP_OK) {
        if (had) ctx->tuned[key] = old;
        return st;
    }
    int32_t dev_status = 0;
    e = cudaMemcpyAsync(&dev_status, st_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && dev_status != 0 && dev_status != TP_E_OVERFLOW) {
        if (had) ctx->tuned[key] = old;
        return status_to_error(ctx, dev_status);
    }
    ctx->tuned[key] = {best_b, best_s, best_p};
    out->block = best_b;
    out->schedule = best_s;
    out->ms = best_ms;
    out->ms_default = def_ms;
    out->candidates = cands;
    out->particles_per_thread = best_p;
    return TP_OK;
}

}  // extern "C"

struct tp_graph {
    tp_ctx* ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long* queue = nullptr;
    ~tp_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (queue) cudaFree(queue);
    }
};

extern "C" {

int tp_boris_graph_create(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, const tp_field* B,
                          const double* u0, const double* dt_i, const double* tend_i, int64_t n, int64_t nslots,
                          double* t_out, double* u_out, int32_t* nsaved, int8_t* retcode, int64_t* nsteps,
                          int32_t* status, tp_graph** out) {
    if (!ctx || !out) return TP_E_ARG;
    *out = nullptr;
    int st = check_boris_desc(ctx, d);
    if (st != TP_OK) return st;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (n <= 0 || nslots < 0) return fail(ctx, TP_E_ARG, "a graph needs n > 0 particles");
    if (!u0 || !nsaved || !retcode || !nsteps || !status || (nslots > 0 && (!t_out || !u_out)))
        return fail(ctx, TP_E_ARG, "null device buffer");
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    if (!adaptive && !dt_i && std::fabs(d->dt) < 10.0 * kEps)
        return fail(ctx, TP_E_ARG, "time step dt is too small, violating min_dt = 10 * eps(typeof(dt))");
    DeviceGuard g(ctx->device);
    BorisArgs a;
    st = prepare_boris_args(ctx, d, E, const_cast<tp_field*>(B), a);
    if (st != TP_OK) return st;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "field table");
    a.n = n;
    a.nslots = nslots;
    a.u0 = u0;
    a.dt_i = dt_i;
    a.tend_i = tend_i;
    a.t_out = t_out;
    a.u_out = u_out;
    a.nsaved = nsaved;
    a.retcode = retcode;
    a.nsteps = nsteps;
    a.status = status;
    LaunchCfg cfg;
    st = plan_boris_launch(ctx, d, a, cfg);
    if (st != TP_OK) return st;
    auto* gr = new tp_graph();
    gr->ctx = ctx;
    if (a.use_queue) {
        e = cudaMalloc((void**)&gr->queue, sizeof(unsigned long long));
        if (e != cudaSuccess) {
            delete gr;
            return cuda_fail(ctx, e, "queue counter");
        }
    }
    cudaStream_t cs = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        if (cs) cudaStreamDestroy(cs);
        delete gr;
        return cuda_fail(ctx, e, "graph capture");
    }
    st = issue_boris_launch(ctx, d, a, cfg, cs, gr->queue);
    cudaError_t ee = cudaStreamEndCapture(cs, &gr->graph);
    cudaStreamDestroy(cs);
    if (st != TP_OK) {
        delete gr;
        return st;
    }
    if (ee == cudaSuccess) ee = cudaGraphInstantiate(&gr->exec, gr->graph, 0);
    if (ee != cudaSuccess) {
        delete gr;
        return cuda_fail(ctx, ee, "graph instantiate");
    }
    *out = gr;
    return TP_OK;
}

int tp_graph_launch(tp_graph* gr, void* stream) {
    if (!gr) return TP_E_ARG;
    DeviceGuard g(gr->ctx->device);
    cudaError_t e = cudaGraphLaunch(gr->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(gr->ctx, e, "graph launch");
    return TP_OK;
}

void tp_graph_destroy(tp_graph* gr) {
    if (!gr) return;
    DeviceGuard g(gr->ctx->device);
    cudaDeviceSynchronize();
    delete gr;
}

int tp_boris_run(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, const tp_field* B,
                 const double* u0, const double* dt_i, const double* tend_i, int64_t n,
                 tp_result** out) {
    if (!ctx || !out) return TP_E_ARG;
    *out = nullptr;
    int st = check_boris_desc(ctx, d);
    if (st != TP_OK) return st;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (n < 0 || (n > 0 && !u0)) return fail(ctx, TP_E_ARG, "bad particle table");
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    int64_t nslots = 0;
    if (!adaptive) {
        // the reference's ArgumentErrors (boris.jl:349-356) before any tracing,
        // in the same pass as the output sizing
        if (d->savestepinterval < 1) return fail(ctx, TP_E_ARG, "cannot size the output");
        const StepScan sc = scan_steps(d, dt_i, tend_i, n);
        if (sc.bad == 1)
            return fail(ctx, TP_E_ARG, "time step dt is too small, violating min_dt = 10 * eps(typeof(dt))");
        if (sc.bad == 2)
            return fail(ctx, TP_E_ARG, "number of iterations nt (" + std::to_string(sc.bad_nt) +
                                           ") exceeds maxiters (" + std::to_string(d->maxiters) + ")");
        nslots = sc.nslots;
    } else {
        st = tp_boris_slots(d, dt_i, tend_i, n, &nslots);
        if (st != TP_OK) return fail(ctx, st, "cannot size the output");
    }
    if (nslots < 0) nslots = 64;  // adaptive without a cap: grown on overflow below
    const int W = 6 + (d->save_fields ? 6 : 0) + (d->save_work ? 4 : 0);
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    tp_result* r = new tp_result();
    for (int attempt = 0; attempt < 2; ++attempt) {
        DBuf u0_d, dt_d, te_d, t_d, u_d, ns_d, rc_d, nst_d, st_d, q_d;
        cudaError_t e = u0_d.alloc((size_t)n * 6 * sizeof(double));
        if (e == cudaSuccess && dt_i) e = dt_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && tend_i) e = te_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess) e = t_d.alloc((size_t)nslots * n * sizeof(double));
        if (e == cudaSuccess) e = u_d.alloc((size_t)nslots * W * n * sizeof(double));
        if (e == cudaSuccess) e = ns_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = rc_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int8_t));
        if (e == cudaSuccess) e = nst_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int64_t));
        if (e == cudaSuccess) e = st_d.alloc(sizeof(int32_t));
        if (e == cudaSuccess) e = q_d.alloc(sizeof(unsigned long long));
        if (e != cudaSuccess) {
            delete r;
            return fail(ctx, TP_E_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
        }
        if (n > 0) e = copy_to_device(ctx, u0_d.p, u0, (size_t)n * 6 * sizeof(double));
        if (e == cudaSuccess && dt_i)
            e = cudaMemcpyAsync(dt_d.p, dt_i, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && tend_i)
            e = cudaMemcpyAsync(te_d.p, tend_i, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(st_d.p, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "input upload");
        }
        BorisArgs a;
        st = prepare_boris_args(ctx, d, E, const_cast<tp_field*>(B), a);
        if (st != TP_OK) {
            delete r;
            return st;
        }
        a.n = n;
        a.nslots = nslots;
        a.u0 = u0_d.as<double>();
        a.dt_i = dt_i ? dt_d.as<double>() : nullptr;
        a.tend_i = tend_i ? te_d.as<double>() : nullptr;
        a.t_out = t_d.as<double>();
        a.u_out = u_d.as<double>();
        a.nsaved = ns_d.as<int32_t>();
        a.retcode = rc_d.as<int8_t>();
        a.nsteps = nst_d.as<int64_t>();
        a.status = st_d.as<int32_t>();
        cudaEvent_t ev0, ev1;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, s);
        if (n > 0) {
            void* obuf = nullptr;
            st = order_particles(ctx, a, s, &obuf);
            if (st == TP_OK) st = launch_boris(ctx, d, a, s, q_d.as<unsigned long long>());
            if (obuf) cudaFreeAsync(obuf, s);
            if (st != TP_OK) {
                cudaEventDestroy(ev0);
                cudaEventDestroy(ev1);
                delete r;
                return st;
            }
        }
        cudaEventRecord(ev1, s);
        int32_t status = 0;
        e = cudaMemcpyAsync(&status, st_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "push kernel");
        }
        r->elapsed_ms = ms;
        if (status == TP_E_OVERFLOW && adaptive && attempt == 0) {
            // saves of an adaptive run are unknown in advance: size exactly and rerun
            std::vector<int32_t> ns(n);
            e = cudaMemcpy(ns.data(), ns_d.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                delete r;
                return cuda_fail(ctx, e, "save counts");
            }
            int64_t mx = 0;
            for (int32_t v : ns) mx = std::max<int64_t>(mx, v);
            nslots = mx;
            continue;
        }
        if (status != 0) {
            delete r;
            return status_to_error(ctx, status);
        }
        st = pack_results(ctx, n, nslots, W, t_d, u_d, ns_d, rc_d, nst_d, r);
        if (st != TP_OK) {
            delete r;
            return st;
        }
        *out = r;
        return TP_OK;
    }
    delete r;
    return fail(ctx, TP_E_OVERFLOW, "save slots exceeded after resizing");
}

}  // extern "C"

namespace {

// One chunk's saves, slot-major in pinned memory (t: [nslots][m], u:
// [nslots * W][m]), into the packed per-trajectory layout of tp_result_copy
// starting at row 0 of t_dst / u_dst; counts clamped to [0, nslots] as the
// device packing does.  Returns the rows written.  Host threads split the
// particles; each walks blocks of 8 particles so that the strided reads
// use whole cache lines.
// Write zeros over n doubles with host threads: the first touch of fresh
// pages (the kernel's page zeroing) happens here, off the copy's path.
void touch_pages(double* p, int64_t n) {
    if (!p || n <= 0) return;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nth = (int)std::min<int64_t>(std::max(1u, std::min(hw, 8u)), (n + (1 << 20) - 1) >> 20);
    std::vector<std::thread> th;
    const int64_t slice = (n + nth - 1) / nth;
    for (int k = 0; k < nth; ++k) {
        const int64_t a = std::min(n, k * slice), b = std::min(n, (k + 1) * slice);
        if (a < b) th.emplace_back([=]() { std::memset(p + a, 0, (size_t)(b - a) * sizeof(double)); });
    }
    for (auto& t : th) t.join();
}

int64_t pack_chunk_host(const double* t_st, const double* u_st, const int32_t* ns, int64_t m, int64_t nslots,
                        int W, double* t_dst, double* u_dst) {
    std::vector<int64_t> off((size_t)m + 1);
    off[0] = 0;
    for (int64_t i = 0; i < m; ++i)
        off[i + 1] = off[i] + std::min<int64_t>(std::max<int32_t>(ns[i], 0), nslots);
    auto part = [&](int64_t a, int64_t b) {
        for (int64_t i0 = a; i0 < b; i0 += 8) {
            const int64_t i1 = std::min(b, i0 + 8);
            for (int64_t s = 0; s < nslots; ++s) {
                for (int64_t i = i0; i < i1; ++i)
                    if (s < off[i + 1] - off[i]) t_dst[off[i] + s] = t_st[s * m + i];
                for (int c = 0; c < W; ++c) {
                    const double* src = u_st + (s * W + c) * m;
                    for (int64_t i = i0; i < i1; ++i)
                        if (s < off[i + 1] - off[i]) u_dst[(off[i] + s) * W + c] = src[i];
                }
            }
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const int nth = (int)std::min<int64_t>(std::max(1u, std::min(hw, 16u)), (m + 8191) / 8192);
    if (nth <= 1) {
        part(0, m);
    } else {
        std::vector<std::thread> th;
        const int64_t slice = ((m + nth - 1) / nth + 7) & ~(int64_t)7;
        for (int k = 0; k < nth; ++k) {
            const int64_t a = std::min(m, k * slice), b = std::min(m, (k + 1) * slice);
            if (a < b) th.emplace_back(part, a, b);
        }
        for (auto& t : th) t.join();
    }
    return off[m];
}

}  // namespace

extern "C" {

// Host-to-host solve with the copy-out overlapped with the push.  One kernel
// runs the whole ensemble; each particle, once its outputs are written,
// counts itself in its chunk (BorisArgs::done).  The queue schedule hands out
// particles in index order, so chunks finish one after another while the
// kernel runs: the host polls the counts and copies each finished chunk's
// slot-major results (two strided copies into pinned staging), then packs
// them into the caller's arrays on host threads.
int tp_boris_run_host(tp_ctx* ctx, const tp_run_desc* d, const tp_field* E, const tp_field* B,
                      const double* u0, const double* dt_i, const double* tend_i, int64_t n, int64_t cap_rows,
                      int32_t* nsaved, int8_t* retcode, int64_t* nsteps, double* t_packed, double* u_packed,
                      int64_t* total, double* elapsed_ms) {
    if (!ctx || !total) return TP_E_ARG;
    *total = 0;
    if (elapsed_ms) *elapsed_ms = 0.0;
    int st = check_boris_desc(ctx, d);
    if (st != TP_OK) return st;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (n < 0 || (n > 0 && (!u0 || !nsaved || !retcode || !nsteps))) return fail(ctx, TP_E_ARG, "bad particle table");
    if (cap_rows < 0 || (cap_rows > 0 && (!t_packed || !u_packed))) return fail(ctx, TP_E_ARG, "bad result buffers");
    const bool adaptive = d->alg == TP_ALG_ADAPTIVE || d->alg == TP_ALG_ADAPTIVE_MULTISTEP;
    int64_t nslots = 0;
    if (!adaptive) {
        // the reference's ArgumentErrors (boris.jl:349-356) before any tracing
        if (d->savestepinterval < 1) return fail(ctx, TP_E_ARG, "cannot size the output");
        const StepScan sc = scan_steps(d, dt_i, tend_i, n);
        if (sc.bad == 1)
            return fail(ctx, TP_E_ARG, "time step dt is too small, violating min_dt = 10 * eps(typeof(dt))");
        if (sc.bad == 2)
            return fail(ctx, TP_E_ARG, "number of iterations nt (" + std::to_string(sc.bad_nt) +
                                           ") exceeds maxiters (" + std::to_string(d->maxiters) + ")");
        nslots = sc.nslots;
    } else {
        st = tp_boris_slots(d, dt_i, tend_i, n, &nslots);
        if (st != TP_OK) return fail(ctx, st, "cannot size the output");
        if (nslots < 0)
            return fail(ctx, TP_E_UNSUPPORTED, "adaptive run without step_cap: the save count is unknown (tp_boris_run)");
    }
    if (n == 0) return TP_OK;
    const int W = 6 + (d->save_fields ? 6 : 0) + (d->save_work ? 4 : 0);
    // chunks of at least 32768 particles, at most 32 of them unless a
    // chunk's staging would exceed 256 MB (the last chunk's copy and packing
    // are what remains after the kernel)
    const int64_t row_bytes = (int64_t)nslots * (W + 1) * 8 + 13;
    int64_t C = std::max<int64_t>(1, std::min<int64_t>(32, n / 32768));
    C = std::max<int64_t>(C, (n * row_bytes + ((int64_t)256 << 20) - 1) / ((int64_t)256 << 20));
    C = std::min<int64_t>(C, n);
    const int64_t cn = (n + C - 1) / C;
    const size_t stage_bytes = (size_t)cn * row_bytes + 64;
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (!ctx->copy_stream) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k)
        if (!ctx->run_ev[k]) e = cudaEventCreate(&ctx->run_ev[k]);
    if (e == cudaSuccess && ctx->done_cap < C) {
        if (ctx->done_pin) cudaFreeHost(ctx->done_pin);
        ctx->done_pin = nullptr;
        ctx->done_cap = 0;
        e = cudaHostAlloc((void**)&ctx->done_pin, (size_t)std::max<int64_t>(C, 64) * sizeof(int32_t),
                          cudaHostAllocDefault);
        if (e == cudaSuccess) ctx->done_cap = std::max<int64_t>(C, 64);
    }
    cudaStream_t s_cp = ctx->copy_stream;
    cudaEvent_t ev0 = ctx->run_ev[0], ev1 = ctx->run_ev[1];
    int32_t* hdone = ctx->done_pin;
    if (e == cudaSuccess && ctx->chunk_pin_bytes < stage_bytes) {
        if (ctx->chunk_pin) cudaFreeHost(ctx->chunk_pin);
        ctx->chunk_pin = nullptr;
        ctx->chunk_pin_bytes = 0;
        e = cudaHostAlloc(&ctx->chunk_pin, stage_bytes, cudaHostAllocDefault);
        if (e == cudaSuccess) ctx->chunk_pin_bytes = stage_bytes;
    }
    if (e != cudaSuccess) {
        return cuda_fail(ctx, e, "pipeline set-up");
    }
    int rc = TP_OK;
    {
        DBuf u0_d, dt_d, te_d, t_d, u_d, ns_d, rc_d, nst_d, st_d, q_d, done_d;
        e = u0_d.alloc((size_t)n * 6 * sizeof(double));
        if (e == cudaSuccess && dt_i) e = dt_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && tend_i) e = te_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess) e = t_d.alloc((size_t)nslots * n * sizeof(double));
        if (e == cudaSuccess) e = u_d.alloc((size_t)nslots * W * n * sizeof(double));
        if (e == cudaSuccess) e = ns_d.alloc((size_t)n * sizeof(int32_t));
        if (e == cudaSuccess) e = rc_d.alloc((size_t)n * sizeof(int8_t));
        if (e == cudaSuccess) e = nst_d.alloc((size_t)n * sizeof(int64_t));
        if (e == cudaSuccess) e = st_d.alloc(sizeof(int32_t));
        if (e == cudaSuccess) e = q_d.alloc(sizeof(unsigned long long));
        if (e == cudaSuccess) e = done_d.alloc((size_t)C * sizeof(int32_t));
        if (e != cudaSuccess) {
            return fail(ctx, TP_E_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
        }
        e = copy_to_device(ctx, u0_d.p, u0, (size_t)n * 6 * sizeof(double));
        if (e == cudaSuccess && dt_i) e = copy_to_device(ctx, dt_d.p, dt_i, (size_t)n * sizeof(double));
        if (e == cudaSuccess && tend_i) e = copy_to_device(ctx, te_d.p, tend_i, (size_t)n * sizeof(double));
        if (e == cudaSuccess) e = cudaMemsetAsync(st_d.p, 0, sizeof(int32_t), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(done_d.p, 0, (size_t)C * sizeof(int32_t), s);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(s);
            return cuda_fail(ctx, e, "input upload");
        }
        BorisArgs a;
        st = prepare_boris_args(ctx, d, E, const_cast<tp_field*>(B), a);
        if (st != TP_OK) {
            cudaStreamSynchronize(s);
            return st;
        }
        a.n = n;
        a.nslots = nslots;
        a.u0 = u0_d.as<double>();
        a.dt_i = dt_i ? dt_d.as<double>() : nullptr;
        a.tend_i = tend_i ? te_d.as<double>() : nullptr;
        a.t_out = t_d.as<double>();
        a.u_out = u_d.as<double>();
        a.nsaved = ns_d.as<int32_t>();
        a.retcode = rc_d.as<int8_t>();
        a.nsteps = nst_d.as<int64_t>();
        a.status = st_d.as<int32_t>();
        // with work rates a post-pass completes the saves: chunks are final
        // only when the whole launch is
        const bool progressive = !a.save_work;
        a.done = progressive ? done_d.as<int32_t>() : nullptr;
        a.done_chunk = cn;
        e = cudaEventRecord(ev0, s);
        // the copy stream's polls and copies come after the counters' reset
        // (pool memory may hold a previous call's counts)
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s_cp, ev0, 0);
        void* obuf = nullptr;
        if (e == cudaSuccess) st = order_particles(ctx, a, s, &obuf);
        if (e == cudaSuccess && st == TP_OK) st = launch_boris(ctx, d, a, s, q_d.as<unsigned long long>());
        if (obuf) cudaFreeAsync(obuf, s);
        if (e == cudaSuccess) e = cudaEventRecord(ev1, s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "push kernel launch");
        else if (st != TP_OK) rc = st;
        // Particles processed in cell order (gridded solves) or saves completed
        // by a post-pass: chunks are final only at the end.  Then the caller's
        // arrays are first touched by host threads while the kernel runs, and
        // the saves are packed on the device and copied through the pinned
        // staging buffers afterwards.
        const bool in_order = progressive && !a.perm;
        int64_t row = 0;
        if (!in_order && rc == TP_OK) {
            std::thread toucher([&]() {
                touch_pages(t_packed, cap_rows);
                touch_pages(u_packed, cap_rows * W);
            });
            e = cudaEventSynchronize(ev1);
            toucher.join();
            DBuf cnt_d, off_d, tmp_d, tp_d, up_d;
            size_t tb = 0;
            if (e == cudaSuccess) e = cnt_d.alloc((size_t)(n + 1) * sizeof(int64_t));
            if (e == cudaSuccess) e = off_d.alloc((size_t)(n + 1) * sizeof(int64_t));
            if (e == cudaSuccess)
                e = scan_offsets(ns_d.as<int32_t>(), n, nslots, cnt_d.as<int64_t>(), off_d.as<int64_t>(), nullptr, &tb, s);
            if (e == cudaSuccess) e = tmp_d.alloc(tb);
            if (e == cudaSuccess)
                e = scan_offsets(ns_d.as<int32_t>(), n, nslots, cnt_d.as<int64_t>(), off_d.as<int64_t>(), tmp_d.p, &tb, s);
            int64_t tot = 0;
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&tot, off_d.as<int64_t>() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                rc = cuda_fail(ctx, e, "result offsets");
            } else if (tot > cap_rows) {
                rc = fail(ctx, TP_E_ARG, "cap_rows is smaller than the number of saves");
            } else {
                e = tp_d.alloc((size_t)std::max<int64_t>(tot, 1) * sizeof(double));
                if (e == cudaSuccess) e = up_d.alloc((size_t)std::max<int64_t>(tot, 1) * W * sizeof(double));
                if (e == cudaSuccess)
                    e = launch_pack_results(t_d.as<double>(), u_d.as<double>(), ns_d.as<int32_t>(),
                                            off_d.as<int64_t>(), n, nslots, W, tp_d.as<double>(), up_d.as<double>(), s);
                if (e == cudaSuccess) e = copy_to_host_on(ctx, s, t_packed, tp_d.p, (size_t)tot * sizeof(double));
                if (e == cudaSuccess) e = copy_to_host_on(ctx, s, u_packed, up_d.p, (size_t)tot * W * sizeof(double));
                if (e == cudaSuccess) e = copy_to_host_on(ctx, s, nsaved, ns_d.p, (size_t)n * sizeof(int32_t));
                if (e == cudaSuccess) e = copy_to_host_on(ctx, s, retcode, rc_d.p, (size_t)n);
                if (e == cudaSuccess) e = copy_to_host_on(ctx, s, nsteps, nst_d.p, (size_t)n * sizeof(int64_t));
                if (e != cudaSuccess) rc = cuda_fail(ctx, e, "result packing");
                else row = tot;
            }
        }
        // otherwise copy each chunk out once all its particles are done
        char* stage = (char*)ctx->chunk_pin;
        for (int64_t k = 0; k < C && rc == TP_OK && in_order; ++k) {
            const int64_t a0 = k * cn, m = std::min(cn, n - a0);
            for (;;) {
                cudaError_t q = cudaEventQuery(ev1);
                if (q == cudaSuccess) break;  // the whole launch is done
                if (q != cudaErrorNotReady) {
                    rc = cuda_fail(ctx, q, "push kernel");
                    break;
                }
                if (progressive) {
                    e = cudaMemcpyAsync(hdone, done_d.p, (size_t)C * sizeof(int32_t), cudaMemcpyDeviceToHost, s_cp);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s_cp);
                    if (e != cudaSuccess) {
                        rc = cuda_fail(ctx, e, "chunk progress");
                        break;
                    }
                    if (hdone[k] >= m) break;
                }
                std::this_thread::sleep_for(std::chrono::microseconds(250));
            }
            if (rc != TP_OK) break;
            double* t_st = (double*)stage;
            double* u_st = t_st + nslots * m;
            int32_t* ns_st = (int32_t*)(u_st + nslots * W * m);
            int64_t* nst_st = (int64_t*)(ns_st + ((m + 1) & ~(int64_t)1));
            int8_t* rc_st = (int8_t*)(nst_st + m);
            e = cudaSuccess;
            if (nslots > 0) {
                e = cudaMemcpy2DAsync(t_st, m * sizeof(double), t_d.as<double>() + a0, n * sizeof(double),
                                      m * sizeof(double), nslots, cudaMemcpyDeviceToHost, s_cp);
                if (e == cudaSuccess)
                    e = cudaMemcpy2DAsync(u_st, m * sizeof(double), u_d.as<double>() + a0, n * sizeof(double),
                                          m * sizeof(double), nslots * W, cudaMemcpyDeviceToHost, s_cp);
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ns_st, ns_d.as<int32_t>() + a0, m * sizeof(int32_t), cudaMemcpyDeviceToHost, s_cp);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(nst_st, nst_d.as<int64_t>() + a0, m * sizeof(int64_t), cudaMemcpyDeviceToHost, s_cp);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(rc_st, rc_d.as<int8_t>() + a0, m, cudaMemcpyDeviceToHost, s_cp);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s_cp);
            if (e != cudaSuccess) {
                rc = cuda_fail(ctx, e, "result copy");
                break;
            }
            int64_t rows = 0;
            for (int64_t i = 0; i < m; ++i) rows += std::min<int64_t>(std::max<int32_t>(ns_st[i], 0), nslots);
            if (row + rows > cap_rows) {
                rc = fail(ctx, TP_E_ARG, "cap_rows is smaller than the number of saves");
                break;
            }
            pack_chunk_host(t_st, u_st, ns_st, m, nslots, W, t_packed + row, u_packed + row * W);
            std::memcpy(nsaved + a0, ns_st, m * sizeof(int32_t));
            std::memcpy(nsteps + a0, nst_st, m * sizeof(int64_t));
            std::memcpy(retcode + a0, rc_st, m);
            row += rows;
        }
        e = cudaStreamSynchronize(s);
        if (rc == TP_OK && e != cudaSuccess) rc = cuda_fail(ctx, e, "push kernel");
        if (rc == TP_OK) {
            int32_t status = 0;
            e = cudaMemcpy(&status, st_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "push status");
            else if (status != 0) rc = status_to_error(ctx, status);
        }
        if (rc == TP_OK) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            if (elapsed_ms) *elapsed_ms = ms;
            *total = row;
        }
        cudaStreamSynchronize(s_cp);
    }
    cudaStreamSynchronize(s);
    return rc;
}

// ---------------------------------------------------------------- guiding centre
int tp_gc_prepare(tp_ctx* ctx, const tp_field* E, const tp_field* B, const double* xv, int64_t n,
                  double q, double m, double t, double* y0_out, double* mu_out) {
    if (!ctx || !E || !B) return fail(ctx, TP_E_ARG, "null argument");
    if (n < 0 || (n > 0 && (!xv || !y0_out || !mu_out))) return fail(ctx, TP_E_ARG, "bad buffers");
    if (n == 0) return TP_OK;
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    DBuf xv_d, y_d, mu_d;
    cudaError_t e = xv_d.alloc((size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess) e = y_d.alloc((size_t)n * 4 * sizeof(double));
    if (e == cudaSuccess) e = mu_d.alloc((size_t)n * sizeof(double));
    if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, "device allocation");
    e = cudaMemcpyAsync(xv_d.p, xv, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, s);
    GCPrepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f.E = E->dev;
    a.f.B = B->dev;
    a.xv = xv_d.as<double>();
    a.n = n;
    a.q = q;
    a.m = m;
    a.t = t;
    a.y0 = y_d.as<double>();
    a.mu = mu_d.as<double>();
    if (e == cudaSuccess) e = launch_gc_prepare(a, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(y0_out, y_d.p, (size_t)n * 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mu_out, mu_d.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "prepare_gc");
    return TP_OK;
}

int tp_gc_to_full(tp_ctx* ctx, const tp_field* E, const tp_field* B, const double* y, const double* mu, int64_t n,
                  double q, double m, double phase, const double* phase_i, double t, double* xv_out) {
    if (!ctx || !E || !B) return fail(ctx, TP_E_ARG, "null argument");
    if (E->ctx != ctx || B->ctx != ctx) return fail(ctx, TP_E_ARG, "fields belong to another context");
    if (n < 0 || (n > 0 && (!y || !mu || !xv_out))) return fail(ctx, TP_E_ARG, "bad buffers");
    if (n == 0) return TP_OK;
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    DBuf y_d, mu_d, ph_d, xv_d;
    cudaError_t e = y_d.alloc((size_t)n * 4 * sizeof(double));
    if (e == cudaSuccess) e = mu_d.alloc((size_t)n * sizeof(double));
    if (e == cudaSuccess && phase_i) e = ph_d.alloc((size_t)n * sizeof(double));
    if (e == cudaSuccess) e = xv_d.alloc((size_t)n * 6 * sizeof(double));
    if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, "device allocation");
    e = cudaMemcpyAsync(y_d.p, y, (size_t)n * 4 * sizeof(double), cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mu_d.p, mu, (size_t)n * sizeof(double), cudaMemcpyDefault, s);
    if (e == cudaSuccess && phase_i)
        e = cudaMemcpyAsync(ph_d.p, phase_i, (size_t)n * sizeof(double), cudaMemcpyDefault, s);
    GCFullArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f.E = E->dev;
    a.f.B = B->dev;
    a.y = y_d.as<double>();
    a.mu = mu_d.as<double>();
    a.phase_i = phase_i ? ph_d.as<double>() : nullptr;
    a.n = n;
    a.q = q;
    a.m = m;
    a.t = t;
    a.phase = phase;
    a.xv = xv_d.as<double>();
    if (e == cudaSuccess) e = launch_gc_to_full(a, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(xv_out, xv_d.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "gc_to_full");
    return TP_OK;
}

int tp_hybrid_run(tp_ctx* ctx, const tp_hybrid_desc* d, const tp_field* E, const tp_field* B, const double* u0,
                  int64_t n, tp_result** out, tp_result** adia) {
    if (!ctx || !d || !out) return fail(ctx, TP_E_ARG, "null argument");
    *out = nullptr;
    if (adia) *adia = nullptr;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (E->ctx != ctx || B->ctx != ctx) return fail(ctx, TP_E_ARG, "fields belong to another context");
    if (n < 0 || (n > 0 && !u0)) return fail(ctx, TP_E_ARG, "bad particle table");
    // AdaptiveHybrid constructor checks (src/hybrid.jl:58-68)
    if (d->check_interval <= 0) return fail(ctx, TP_E_ARG, "check_interval must be positive.");
    if (!(d->threshold_gc_to_fo >= d->threshold_fo_to_gc))
        return fail(ctx, TP_E_ARG, "threshold_gc_to_fo must be >= threshold_fo_to_gc for hysteresis.");
    if (d->adiabaticity < TP_ADIA_CURVATURE || d->adiabaticity > TP_ADIA_JACOBIAN)
        return fail(ctx, TP_E_ARG, "adiabaticity must be one of :curvature, :gradB, :both, :jacobian.");
    if (d->savestepinterval < 1) return fail(ctx, TP_E_ARG, "savestepinterval must be >= 1");
    if (d->maxiters < 0) return fail(ctx, TP_E_ARG, "maxiters must be >= 0");
    if (d->block < 0 || d->block > 256 || (d->block % 32) != 0)
        return fail(ctx, TP_E_ARG, "block must be 0 or a multiple of 32 up to 256");
    const bool want_adia = adia && d->save_adiabaticity;
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    int64_t nslots = 64, aslots = want_adia ? 64 : 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        DBuf u0_d, t_d, u_d, ns_d, rc_d, nst_d, at_d, av_d, na_d, st_d;
        cudaError_t e = u0_d.alloc((size_t)std::max<int64_t>(n, 1) * 6 * sizeof(double));
        if (e == cudaSuccess) e = t_d.alloc((size_t)std::max<int64_t>(nslots * n, 1) * sizeof(double));
        if (e == cudaSuccess) e = u_d.alloc((size_t)std::max<int64_t>(nslots * n, 1) * 6 * sizeof(double));
        if (e == cudaSuccess) e = ns_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = rc_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int8_t));
        if (e == cudaSuccess) e = nst_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int64_t));
        if (e == cudaSuccess && want_adia) e = at_d.alloc((size_t)std::max<int64_t>(aslots * n, 1) * sizeof(double));
        if (e == cudaSuccess && want_adia)
            e = av_d.alloc((size_t)std::max<int64_t>(aslots * n, 1) * 2 * sizeof(double));
        if (e == cudaSuccess && want_adia) e = na_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = st_d.alloc(sizeof(int32_t));
        if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
        if (n > 0) e = copy_to_device(ctx, u0_d.p, u0, (size_t)n * 6 * sizeof(double));
        if (e == cudaSuccess) e = cudaMemsetAsync(st_d.p, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "input upload");
        HybridArgs a;
        std::memset(&a, 0, sizeof(a));
        a.f.E = E->dev;
        a.f.B = B->dev;
        a.term = dev_term(d->term);
        a.t0 = d->t0;
        a.t1 = d->t1;
        a.q2m = d->q2m;
        a.m = d->m;
        a.th_gc_fo = d->threshold_gc_to_fo;
        a.th_fo_gc = d->threshold_fo_to_gc;
        a.dtmin = d->dtmin;
        a.dtmax = d->dtmax;
        a.safety_fo = d->safety_fo;
        a.abstol = d->abstol;
        a.reltol = d->reltol;
        a.maxiters = d->maxiters;
        a.check = d->check_interval;
        a.ssi = d->savestepinterval;
        a.adia_mode = d->adiabaticity;
        a.save_adia = want_adia ? 1 : 0;
        a.save_start = d->save_start;
        a.save_end = d->save_end;
        a.save_everystep = d->save_everystep;
        a.n = n;
        a.nslots = nslots;
        a.aslots = aslots;
        a.u0 = u0_d.as<double>();
        a.t_out = t_d.as<double>();
        a.u_out = u_d.as<double>();
        a.nsaved = ns_d.as<int32_t>();
        a.retcode = rc_d.as<int8_t>();
        a.nsteps = nst_d.as<int64_t>();
        a.at_out = at_d.as<double>();
        a.av_out = av_d.as<double>();
        a.nadia = na_d.as<int32_t>();
        a.status = st_d.as<int32_t>();
        double budget = d->budget_s > 0 ? d->budget_s : 600.0;
        a.budget_ns = (uint64_t)(budget * 1e9);
        e = prime_hybrid(a);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel load");
        cudaEvent_t ev0, ev1;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, s);
        e = launch_hybrid(a, d->block, s);
        cudaEventRecord(ev1, s);
        int32_t status = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&status, st_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "hybrid kernel");
        if (status == TP_E_OVERFLOW && attempt == 0) {
            // save and check counts are unknown in advance: size exactly and rerun
            std::vector<int32_t> ns(n), na(want_adia ? n : 0);
            e = cudaMemcpy(ns.data(), ns_d.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (e == cudaSuccess && want_adia)
                e = cudaMemcpy(na.data(), na_d.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "save counts");
            for (int32_t v : ns) nslots = std::max<int64_t>(nslots, v);
            for (int32_t v : na) aslots = std::max<int64_t>(aslots, v);
            continue;
        }
        if (status != 0) return status_to_error(ctx, status);
        DBuf arc_d, anst_d;
        if (want_adia) {
            e = arc_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int8_t));
            if (e == cudaSuccess) e = anst_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int64_t));
            if (e == cudaSuccess && n > 0)
                e = cudaMemcpyAsync(arc_d.p, rc_d.p, (size_t)n * sizeof(int8_t), cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess && n > 0)
                e = cudaMemcpyAsync(anst_d.p, nst_d.p, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "adiabaticity result");
        }
        tp_result* r = new tp_result();
        int st = pack_results(ctx, n, nslots, 6, t_d, u_d, ns_d, rc_d, nst_d, r);
        if (st != TP_OK) {
            delete r;
            return st;
        }
        r->elapsed_ms = ms;
        if (want_adia) {
            tp_result* ra = new tp_result();
            st = pack_results(ctx, n, aslots, 2, at_d, av_d, na_d, arc_d, anst_d, ra);
            if (st != TP_OK) {
                delete ra;
                delete r;
                return st;
            }
            ra->elapsed_ms = ms;
            *adia = ra;
        }
        *out = r;
        return TP_OK;
    }
    return fail(ctx, TP_E_OVERFLOW, "save slots exceeded after resizing");
}


namespace {
bool is_device_ptr(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}
}  // namespace

// Inputs of the detector entry points on the device: host arrays are
// copied (their total number of saves from the host nsaved), device arrays
// are used in place.
struct DetInputs {
    DBuf t_d, u_d, ns_d, w_d, surf_d;
    const double *t = nullptr, *u = nullptr, *w = nullptr;
    const int32_t* ns = nullptr;
    const tp_surface* surf = nullptr;
};

int det_inputs(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved, int64_t n,
               const tp_surface* surfaces, int32_t nsurf, const double* weights, bool flux, DetInputs& in) {
    if (width < 6) return fail(ctx, TP_E_ARG, "width must be >= 6 (x, v first)");
    if (n < 0 || nsurf < 1 || !surfaces) return fail(ctx, TP_E_ARG, "need n >= 0 trajectories and a surface");
    if (n > 0 && (!t || !u || !nsaved)) return fail(ctx, TP_E_ARG, "null trajectory buffer");
    for (int j = 0; j < nsurf; ++j) {
        const tp_surface& S = surfaces[j];
        if (S.kind < TP_SURF_PLANE || S.kind > TP_SURF_SPHERE) return fail(ctx, TP_E_ARG, "unknown surface kind");
        if (flux && S.kind == TP_SURF_PLANE) return fail(ctx, TP_E_ARG, "fluxes need a disk or a sphere (an area)");
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = in.surf_d.alloc((size_t)nsurf * sizeof(tp_surface));
    if (e == cudaSuccess) e = cudaMemcpyAsync(in.surf_d.p, surfaces, (size_t)nsurf * sizeof(tp_surface),
                                              cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "surfaces");
    in.surf = in.surf_d.as<tp_surface>();
    if (n == 0) return TP_OK;
    if (is_device_ptr(u)) {
        in.t = t;
        in.u = u;
        in.ns = nsaved;
        if (weights && !is_device_ptr(weights)) {
            e = in.w_d.alloc((size_t)n * sizeof(double));
            if (e == cudaSuccess) e = copy_to_device(ctx, in.w_d.p, weights, (size_t)n * sizeof(double));
            if (e != cudaSuccess) return cuda_fail(ctx, e, "weights");
            in.w = in.w_d.as<double>();
        } else {
            in.w = weights;
        }
        return TP_OK;
    }
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) total += nsaved[i] > 0 ? nsaved[i] : 0;
    e = in.t_d.alloc((size_t)std::max<int64_t>(total, 1) * sizeof(double));
    if (e == cudaSuccess) e = in.u_d.alloc((size_t)std::max<int64_t>(total, 1) * width * sizeof(double));
    if (e == cudaSuccess) e = in.ns_d.alloc((size_t)n * sizeof(int32_t));
    if (e == cudaSuccess && weights) e = in.w_d.alloc((size_t)n * sizeof(double));
    if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, "device allocation");
    e = copy_to_device(ctx, in.t_d.p, t, (size_t)total * sizeof(double));
    if (e == cudaSuccess) e = copy_to_device(ctx, in.u_d.p, u, (size_t)total * width * sizeof(double));
    if (e == cudaSuccess) e = copy_to_device(ctx, in.ns_d.p, nsaved, (size_t)n * sizeof(int32_t));
    if (e == cudaSuccess && weights) e = copy_to_device(ctx, in.w_d.p, weights, (size_t)n * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trajectory upload");
    in.t = in.t_d.as<double>();
    in.u = in.u_d.as<double>();
    in.ns = in.ns_d.as<int32_t>();
    in.w = weights ? in.w_d.as<double>() : nullptr;
    return TP_OK;
}

int tp_detect_fluxes(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved, int64_t n,
                     const tp_surface* surfaces, int32_t nsurf, const double* weights, double weight,
                     double* n_flux, double* v_flux) {
    if (!ctx || !n_flux || !v_flux) return fail(ctx, TP_E_ARG, "null argument");
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    DetInputs in;
    int st = det_inputs(ctx, t, u, width, nsaved, n, surfaces, nsurf, weights, true, in);
    if (st != TP_OK) return st;
    std::vector<double> tot((size_t)nsurf * 4, 0.0);
    if (n > 0) {
        DBuf tot_d;
        cudaError_t e = tot_d.alloc((size_t)nsurf * 4 * sizeof(double));
        if (e == cudaSuccess)
            e = launch_detect(0, in.t, in.u, width, in.ns, n, in.surf, nsurf, in.w, weight, tot_d.as<double>(),
                              nullptr, nullptr, nullptr, ctx->stream);
        if (e == cudaSuccess) e = copy_to_host(ctx, tot.data(), tot_d.p, tot.size() * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "detector fluxes");
    }
    // get_particle_flux(es): sums times inv(area) (Meshes: pi r^2, 4 pi r^2)
    const double pi = 3.141592653589793;
    for (int j = 0; j < nsurf; ++j) {
        const double r = surfaces[j].radius;
        const double area = surfaces[j].kind == TP_SURF_SPHERE ? (4.0 * pi) * (r * r) : pi * (r * r);
        const double inv_area = 1.0 / area;
        n_flux[j] = tot[4 * j] * inv_area;
        for (int c = 0; c < 3; ++c) v_flux[3 * j + c] = tot[4 * j + 1 + c] * inv_area;
    }
    return TP_OK;
}

int tp_detect_crossings(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                        int64_t n, const tp_surface* surfaces, int32_t nsurf, const double* weights, double weight,
                        int64_t* counts, double* rows) {
    if (!ctx || !counts) return fail(ctx, TP_E_ARG, "null argument");
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    DetInputs in;
    int st = det_inputs(ctx, t, u, width, nsaved, n, surfaces, nsurf, weights, false, in);
    if (st != TP_OK) return st;
    for (int j = 0; j < nsurf; ++j) counts[j] = 0;
    if (n == 0) return TP_OK;
    double* rows_d = nullptr;
    cudaError_t e = launch_detect(1, in.t, in.u, width, in.ns, n, in.surf, nsurf, in.w, weight, nullptr, counts,
                                  rows ? &rows_d : nullptr, nullptr, ctx->stream);
    if (e == cudaSuccess && rows) {
        int64_t total = 0;
        for (int j = 0; j < nsurf; ++j) total += counts[j];
        e = copy_to_host(ctx, rows, rows_d, (size_t)total * 4 * sizeof(double));
    }
    if (rows_d) cudaFreeAsync(rows_d, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "detector crossings");
    return TP_OK;
}

int tp_detect_first_crossing(tp_ctx* ctx, const double* t, const double* u, int32_t width, const int32_t* nsaved,
                             int64_t n, const tp_surface* surface, double* out) {
    if (!ctx || !out) return fail(ctx, TP_E_ARG, "null argument");
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    DetInputs in;
    int st = det_inputs(ctx, t, u, width, nsaved, n, surface, 1, nullptr, false, in);
    if (st != TP_OK) return st;
    if (n == 0) return TP_OK;
    const bool o_dev = is_device_ptr(out);
    DBuf o_d;
    cudaError_t e = o_dev ? cudaSuccess : o_d.alloc((size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess)
        e = launch_detect(2, in.t, in.u, width, in.ns, n, in.surf, 1, nullptr, 0.0, nullptr, nullptr, nullptr,
                          o_dev ? out : o_d.as<double>(), ctx->stream);
    if (e == cudaSuccess)
        e = o_dev ? cudaStreamSynchronize(ctx->stream) : copy_to_host(ctx, out, o_d.p, (size_t)n * 6 * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "first crossing");
    return TP_OK;
}

int tp_eval_points(tp_ctx* ctx, const tp_points_desc* d, const tp_field* E, const tp_field* B,
                   const double* u, const double* t, int64_t n, double* out) {
    return tp_eval_points_params(ctx, d, E, B, u, t, nullptr, nullptr, nullptr, nullptr, n, out);
}

int tp_eval_points_params(tp_ctx* ctx, const tp_points_desc* d, const tp_field* E, const tp_field* B,
                          const double* u, const double* t, const double* q2m_i, const double* m_i,
                          const double* q_i, const double* mu_i, int64_t n, double* out) {
    if (!ctx || !d || !E || !B) return fail(ctx, TP_E_ARG, "null argument");
    if (d->kind != TP_POINTS_FULL_ORBIT && d->kind != TP_POINTS_GC) return fail(ctx, TP_E_ARG, "unknown state kind");
    if (d->want < 1 || d->want > 3) return fail(ctx, TP_E_ARG, "want must select fields (1), work (2) or both (3)");
    const int minw = d->kind == TP_POINTS_GC ? 4 : 6;
    if (d->stride < minw) return fail(ctx, TP_E_ARG, "stride is shorter than a state");
    if (n < 0 || (n > 0 && (!u || !t || !out))) return fail(ctx, TP_E_ARG, "bad buffers");
    if (E->ctx != ctx || B->ctx != ctx) return fail(ctx, TP_E_ARG, "fields belong to another context");
    if (n == 0) return TP_OK;
    const int wout = 6 * (d->want & 1) + 4 * ((d->want >> 1) & 1);
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    const size_t ub = (size_t)n * d->stride * sizeof(double), tb = (size_t)n * sizeof(double),
                 ob = (size_t)n * wout * sizeof(double);
    // device-resident arguments are used in place
    const bool u_dev = is_device_ptr(u), t_dev = is_device_ptr(t), o_dev = is_device_ptr(out);
    DBuf u_d, t_d, o_d;
    cudaError_t e = cudaSuccess;
    if (!u_dev) e = u_d.alloc(ub);
    if (e == cudaSuccess && !t_dev) e = t_d.alloc(tb);
    if (e == cudaSuccess && !o_dev) e = o_d.alloc(ob);
    // per-point parameters: used in place when already on the device
    const double* par[4] = {q2m_i, m_i, q_i, mu_i};
    const double* par_d[4] = {nullptr, nullptr, nullptr, nullptr};
    DBuf par_buf[4];
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        if (!par[k]) continue;
        if (is_device_ptr(par[k])) {
            par_d[k] = par[k];
            continue;
        }
        e = par_buf[k].alloc(tb);
        if (e == cudaSuccess) e = copy_to_device(ctx, par_buf[k].p, par[k], tb);
        par_d[k] = par_buf[k].as<double>();
    }
    if (e != cudaSuccess) return fail(ctx, TP_E_NOMEM, "device allocation");
    if (!u_dev) e = copy_to_device(ctx, u_d.p, u, ub);
    if (e == cudaSuccess && !t_dev) e = copy_to_device(ctx, t_d.p, t, tb);
    PointsArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f.E = E->dev;
    a.f.B = B->dev;
    a.u = u_dev ? u : u_d.as<double>();
    a.t = t_dev ? t : t_d.as<double>();
    a.n = n;
    a.stride = d->stride;
    a.want = d->want;
    a.wout = wout;
    a.kind = d->kind;
    a.q2m = d->q2m;
    a.m = d->m;
    a.q = d->q;
    a.mu = d->mu;
    a.q2m_i = par_d[0];
    a.m_i = par_d[1];
    a.q_i = par_d[2];
    a.mu_i = par_d[3];
    a.out = o_dev ? out : o_d.as<double>();
    if (e == cudaSuccess) e = launch_eval_points(a, ctx->stream);
    if (e == cudaSuccess) e = o_dev ? cudaStreamSynchronize(ctx->stream) : copy_to_host(ctx, out, o_d.p, ob);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "eval_points");
    return TP_OK;
}

int tp_gc_run(tp_ctx* ctx, const tp_gc_desc* d, const tp_field* E, const tp_field* B,
              const double* y0, const double* q_i, const double* q2m_i, const double* mu_i,
              const double* dt_i, const double* tend_i, int64_t n, tp_result** out) {
    if (!ctx || !out || !d) return fail(ctx, TP_E_ARG, "null argument");
    *out = nullptr;
    if (!E || !B) return fail(ctx, TP_E_ARG, "null field");
    if (n < 0 || (n > 0 && !y0)) return fail(ctx, TP_E_ARG, "bad particle table");
    if (d->alg != TP_GC_RK4 && d->alg != TP_GC_RK45) return fail(ctx, TP_E_UNSUPPORTED, "unknown GC algorithm");
    if (d->precision != TP_GC_PREC_FP64 && d->precision != TP_GC_PREC_FP32RHS)
        return fail(ctx, TP_E_UNSUPPORTED, "unknown GC precision");
    if (d->block < 0 || d->block > 256 || (d->block % 32) != 0)
        return fail(ctx, TP_E_ARG, "block must be 0 or a multiple of 32 up to 256");
    // _prepare_gc, src/gc/gc_solver.jl:187-231
    double ttotal = d->t1 - d->t0;
    int64_t nt = 0;
    if (!d->dt_given) {
        if (d->alg == TP_GC_RK4) return fail(ctx, TP_E_ARG, "dt must be provided for fixed step solver :rk4");
    } else {
        int sdt = (d->dt > 0) - (d->dt < 0), stt = (ttotal > 0) - (ttotal < 0);
        if (d->alg == TP_GC_RK4 && sdt != stt && ttotal != 0)
            return fail(ctx, TP_E_ARG, "dt must have the same sign as tspan[2] - tspan[1] for fixed step solver :rk4");
        nt = jl_round_h(ttotal / d->dt);
        if (d->alg == TP_GC_RK4 && nt > d->maxiters) nt = d->maxiters;
    }
    if (d->savestepinterval < 1) return fail(ctx, TP_E_ARG, "savestepinterval must be >= 1");
    int64_t nout = 0;
    if (d->save_start) nout += 1;
    if (d->alg == TP_GC_RK4 && d->save_everystep) {
        int64_t steps = nt / d->savestepinterval;
        bool last_is_step = (nt > 0) && (nt % d->savestepinterval == 0);
        nout += steps;
        if (!d->save_end && last_is_step) nout -= 1;
        if (d->save_end && !last_is_step) nout += 1;
    } else if (d->alg == TP_GC_RK4 && d->save_end) {
        nout += 1;
    }
    if ((dt_i || tend_i) && d->alg == TP_GC_RK4) {
        // per-particle dt / tspan (extension): the same checks and counts per particle
        nout = 0;
        for (int64_t i = 0; i < n; ++i) {
            double dti = dt_i ? dt_i[i] : d->dt;
            double t1i = tend_i ? tend_i[i] : d->t1;
            double tt = t1i - d->t0;
            int sdt = (dti > 0) - (dti < 0), stt = (tt > 0) - (tt < 0);
            if (sdt != stt && tt != 0)
                return fail(ctx, TP_E_ARG, "dt must have the same sign as tspan[2] - tspan[1] for fixed step solver :rk4");
            int64_t nti = jl_round_h(tt / dti);
            if (nti > d->maxiters) nti = d->maxiters;
            int64_t no = d->save_start ? 1 : 0;
            if (d->save_everystep) {
                int64_t steps = nti / d->savestepinterval;
                bool last_is_step = (nti > 0) && (nti % d->savestepinterval == 0);
                no += steps;
                if (!d->save_end && last_is_step) no -= 1;
                if (d->save_end && !last_is_step) no += 1;
            } else if (d->save_end) {
                no += 1;
            }
            nout = std::max(nout, no);
        }
    }
    int64_t nslots = d->alg == TP_GC_RK4 ? std::max<int64_t>(nout, 0) : 64;
    if (d->alg == TP_GC_RK45 && !d->save_everystep) nslots = 2;
    const int W = 4 + (d->save_fields ? 6 : 0) + (d->save_work ? 4 : 0);
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    cudaStream_t s = ctx->stream;
    tp_result* r = new tp_result();
    for (int attempt = 0; attempt < 2; ++attempt) {
        DBuf y_d, q_d, q2m_d, mu_d, dt_d, te_d, t_d, u_d, ns_d, rc_d, nst_d, st_d, qq_d;
        cudaError_t e = y_d.alloc((size_t)n * 4 * sizeof(double));
        if (e == cudaSuccess && dt_i) e = dt_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && tend_i) e = te_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && q_i) e = q_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && q2m_i) e = q2m_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess && mu_i) e = mu_d.alloc((size_t)n * sizeof(double));
        if (e == cudaSuccess) e = t_d.alloc((size_t)nslots * n * sizeof(double));
        if (e == cudaSuccess) e = u_d.alloc((size_t)nslots * W * n * sizeof(double));
        if (e == cudaSuccess) e = ns_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = rc_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int8_t));
        if (e == cudaSuccess) e = nst_d.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(int64_t));
        if (e == cudaSuccess) e = st_d.alloc(sizeof(int32_t));
        if (e == cudaSuccess) e = qq_d.alloc(sizeof(unsigned long long));
        if (e != cudaSuccess) {
            delete r;
            return fail(ctx, TP_E_NOMEM, "device allocation");
        }
        if (n > 0) e = copy_to_device(ctx, y_d.p, y0, (size_t)n * 4 * sizeof(double));
        if (e == cudaSuccess && q_i) e = cudaMemcpyAsync(q_d.p, q_i, (size_t)n * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && q2m_i) e = cudaMemcpyAsync(q2m_d.p, q2m_i, (size_t)n * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && mu_i) e = cudaMemcpyAsync(mu_d.p, mu_i, (size_t)n * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && dt_i) e = cudaMemcpyAsync(dt_d.p, dt_i, (size_t)n * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && tend_i) e = cudaMemcpyAsync(te_d.p, tend_i, (size_t)n * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(st_d.p, 0, sizeof(int32_t), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(qq_d.p, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "input upload");
        }
        GCArgs a;
        std::memset(&a, 0, sizeof(a));
        a.f.E = E->dev;
        a.f.B = B->dev;
        a.term = dev_term(d->term);
        a.alg = d->alg;
        a.precision = d->precision;
        a.save_fields = d->save_fields;
        a.save_work = d->save_work;
        a.dt_given = d->dt_given;
        a.save_start = d->save_start;
        a.save_end = d->save_end;
        a.save_everystep = d->save_everystep;
        a.t0 = d->t0;
        a.t1 = d->t1;
        a.dt = d->dt;
        a.q = d->q;
        a.q2m = d->q2m;
        a.mu = d->mu;
        a.abstol = d->abstol;
        a.reltol = d->reltol;
        a.ssi = d->savestepinterval;
        a.maxiters = d->maxiters;
        a.nt = nt;
        a.nout = nout;
        a.n = n;
        a.nslots = nslots;
        a.y0 = y_d.as<double>();
        a.q_i = q_i ? q_d.as<double>() : nullptr;
        a.q2m_i = q2m_i ? q2m_d.as<double>() : nullptr;
        a.mu_i = mu_i ? mu_d.as<double>() : nullptr;
        a.dt_i = dt_i ? dt_d.as<double>() : nullptr;
        a.tend_i = tend_i ? te_d.as<double>() : nullptr;
        a.t_out = t_d.as<double>();
        a.u_out = u_d.as<double>();
        a.nsaved = ns_d.as<int32_t>();
        a.retcode = rc_d.as<int8_t>();
        a.nsteps = nst_d.as<int64_t>();
        a.status = st_d.as<int32_t>();
        a.queue = qq_d.as<unsigned long long>();
        a.use_queue = d->alg == TP_GC_RK45 || d->term.flags != 0;
        double budget = d->budget_s > 0 ? d->budget_s : 600.0;
        a.budget_ns = (uint64_t)(budget * 1e9);
        int block = d->block > 0 ? d->block : 128;
        LaunchCfg cfg;
        int occ = a.use_queue ? occupancy_gc(a, block) : 0;
        int st = pick_launch(ctx, n, block, a.use_queue, occ, cfg);
        if (st != TP_OK) {
            delete r;
            return st;
        }
        e = prime_gc(a);
        if (e == cudaSuccess && a.save_work) e = prime_fill_work();
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "kernel load");
        }
        cudaEvent_t ev0, ev1;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, s);
        if (n > 0) e = launch_gc(a, cfg, s);
        if (e == cudaSuccess && n > 0 && a.save_work && a.nslots > 0) {
            WorkFillArgs w;
            std::memset(&w, 0, sizeof(w));
            w.f = a.f;
            w.t_out = a.t_out;
            w.u_out = a.u_out;
            w.nsaved = a.nsaved;
            w.n = a.n;
            w.nslots = a.nslots;
            w.c0 = a.save_fields ? 10 : 4;
            w.W = w.c0 + 4;
            w.gc = 1;
            w.q = a.q;
            w.q2m = a.q2m;
            w.mu = a.mu;
            w.q_i = a.q_i;
            w.q2m_i = a.q2m_i;
            w.mu_i = a.mu_i;
            e = launch_fill_work(w, s);
        }
        cudaEventRecord(ev1, s);
        int32_t status = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&status, st_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "guiding-centre kernel");
        }
        r->elapsed_ms = ms;
        if (status == TP_E_OVERFLOW && d->alg == TP_GC_RK45 && attempt == 0) {
            std::vector<int32_t> ns(n);
            e = cudaMemcpy(ns.data(), ns_d.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                delete r;
                return cuda_fail(ctx, e, "save counts");
            }
            int64_t mx = 0;
            for (int32_t v : ns) mx = std::max<int64_t>(mx, v);
            nslots = mx;
            continue;
        }
        if (status != 0) {
            delete r;
            return status_to_error(ctx, status);
        }
        st = pack_results(ctx, n, nslots, W, t_d, u_d, ns_d, rc_d, nst_d, r);
        if (st != TP_OK) {
            delete r;
            return st;
        }
        *out = r;
        return TP_OK;
    }
    delete r;
    return fail(ctx, TP_E_OVERFLOW, "save slots exceeded after resizing");
}

// ---------------------------------------------------------------- results
int tp_result_info(const tp_result* r, int64_t* n, int32_t* width, int64_t* total) {
    if (!r) return TP_E_ARG;
    if (n) *n = r->n;
    if (width) *width = r->width;
    if (total) *total = r->total;
    return TP_OK;
}

int tp_result_copy(const tp_result* r, int32_t* nsaved, int8_t* retcode, int64_t* nsteps,
                   double* t_packed, double* u_packed) {
    if (!r) return TP_E_ARG;
    if (r->n == 0) return TP_OK;
    tp_ctx* ctx = r->ctx;
    DeviceGuard g(ctx->device);
    cudaError_t e = cudaSuccess;
    if (nsaved) e = copy_to_host(ctx, nsaved, r->nsaved, (size_t)r->n * sizeof(int32_t));
    if (e == cudaSuccess && retcode) e = copy_to_host(ctx, retcode, r->retcode, (size_t)r->n * sizeof(int8_t));
    if (e == cudaSuccess && nsteps) e = copy_to_host(ctx, nsteps, r->nsteps, (size_t)r->n * sizeof(int64_t));
    if (e == cudaSuccess && t_packed && r->total)
        e = copy_to_host(ctx, t_packed, r->t, (size_t)r->total * sizeof(double));
    if (e == cudaSuccess && u_packed && r->total)
        e = copy_to_host(ctx, u_packed, r->u, (size_t)r->total * r->width * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
    return TP_OK;
}

int tp_result_elapsed_ms(const tp_result* r, double* ms) {
    if (!r || !ms) return TP_E_ARG;
    *ms = r->elapsed_ms;
    return TP_OK;
}

void tp_result_destroy(tp_result* r) {
    if (!r) return;
    if (r->ctx) {
        DeviceGuard g(r->ctx->device);
        delete r;
        return;
    }
    delete r;
}

}  // extern "C"

// ============================================================ adjoint
struct tp_tape {
    tp_ctx* ctx = nullptr;
    const tp_field* E = nullptr;
    const tp_field* B = nullptr;
    uint64_t E_id = 0, B_id = 0;
    AdjArgs A{};
    int fk = 0;
    LaunchCfg cfg{};
    int64_t nodes_E = 0, nodes_B = 0;
    float* d_ckpt = nullptr;
    double* d_u0 = nullptr;
    float* d_rec = nullptr;
    float4* d_geb = nullptr;
    float4* d_gE = nullptr;
    float4* d_gB = nullptr;
    double* d_gparam = nullptr;
    int32_t* d_need = nullptr;
    float* d_lam = nullptr;
    int G = 0;  // scale exponent of the node-gradient tables, kept for the next pass
    int64_t bytes = 0;
    ~tp_tape() {
        for (void* q : {(void*)d_ckpt, (void*)d_u0, (void*)d_rec, (void*)d_geb, (void*)d_gE, (void*)d_gB,
                        (void*)d_gparam, (void*)d_need, (void*)d_lam})
            if (q) cudaFree(q);
    }
};

namespace {

bool field_static(const tp_field* f) {
    if (f->desc.kind == TP_FIELD_SERIES) return false;
    if (f->desc.kind != TP_FIELD_AFFINE && f->desc.kind != TP_FIELD_QUADRATIC) return true;
    return f->desc.rate[0] == 0.0 && f->desc.rate[1] == 0.0 && f->desc.rate[2] == 0.0;
}

template <class T>
cudaError_t tape_alloc(tp_tape* t, T** p, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) t->bytes += (int64_t)bytes;
    return e;
}

// Validate, build the launch block and allocate the checkpoint tape.
int adjoint_prepare(tp_ctx* ctx, const tp_adj_desc* d, const tp_field* E, const tp_field* B, int64_t n,
                    tp_tape** out) {
    if (!ctx || !d || !E || !B || !out) return fail(ctx, TP_E_ARG, "null argument");
    *out = nullptr;
    const tp_run_desc* r = &d->run;
    int st = check_boris_desc(ctx, r);
    if (st != TP_OK) return st;
    if (r->alg != TP_ALG_BORIS) return fail(ctx, TP_E_UNSUPPORTED, "the adjoint covers the fixed-step Boris map");
    if (r->precision != TP_PREC_FP32C)
        return fail(ctx, TP_E_UNSUPPORTED, "the adjoint runs in TP_PREC_FP32C arithmetic");
    if (r->term.flags != 0) return fail(ctx, TP_E_UNSUPPORTED, "the adjoint takes no termination predicate");
    if (!field_static(E) || !field_static(B))
        return fail(ctx, TP_E_UNSUPPORTED, "the adjoint needs static fields");
    if (E->dev.general || B->dev.general)
        return fail(ctx, TP_E_UNSUPPORTED, "the adjoint covers trilinear uniform Cartesian grids");
    if (E->desc.kind == TP_FIELD_QUADRATIC || B->desc.kind == TP_FIELD_QUADRATIC)
        return fail(ctx, TP_E_UNSUPPORTED, "the adjoint does not cover quadratic fields");
    if (d->checkpoint_every < 0) return fail(ctx, TP_E_ARG, "checkpoint_every must be >= 0 (0: automatic)");
    if (n < 0) return fail(ctx, TP_E_ARG, "negative particle count");
    if (E->ctx != ctx || B->ctx != ctx) return fail(ctx, TP_E_ARG, "fields belong to another context");
    double dt = r->dt;
    if (!(std::fabs(dt) >= 10.0 * kEps) || !std::isfinite(dt))
        return fail(ctx, TP_E_ARG, "dt is too small (|dt| < 10 eps)");
    int64_t nt = jl_round_h((r->t1 - r->t0) / dt);
    if (nt < 0) return fail(ctx, TP_E_ARG, "the adjoint needs (t1 - t0) / dt >= 0");
    if (nt > r->maxiters) return fail(ctx, TP_E_ARG, "nt exceeds maxiters");
    DeviceGuard g(ctx->device);
    auto* t = new tp_tape();
    t->ctx = ctx;
    t->E = E;
    t->B = B;
    t->E_id = E->id;
    t->B_id = B->id;
    AdjArgs& A = t->A;
    st = prepare_boris_args(ctx, r, E, const_cast<tp_field*>(B), A.a);
    if (st != TP_OK) {
        delete t;
        return st;
    }
    A.a.n = n;
    A.nt = nt;
    t->fk = adjoint_field_config(A.a.f);
    int64_t K = d->checkpoint_every;
    if (K == 0) {
        // Automatic: an interleaved E/B grid takes 2-step segments (the
        // one-kernel backward) when their checkpoints fit in half of the free
        // device memory, else 64-step segments; other fields take 64.
        K = 64;
        size_t free_b = 0, total_b = 0;
        if (t->fk == FK_EBGRID && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
            (double)((nt + 1) / 2 + 1) * kAdjCkWords * 4.0 * (double)n <= 0.5 * (double)free_b)
            K = 2;
    }
    A.K = K < nt ? K : (nt > 0 ? nt : 1);
    A.S = nt > 0 ? (nt + A.K - 1) / A.K : 1;
    // final save of _boris_loop! at it = nt: t_final = t1, dt_final = t1 - (t0 + (nt - 1/2) dt)
    A.dt_final = r->t1 - std::fma((double)nt - 0.5, dt, r->t0);
    t->nodes_E = E->nodes;
    t->nodes_B = B->nodes;
    // blocks of at most 128 threads (the segment kernels' launch bounds)
    st = pick_launch(ctx, n, r->block > 0 && r->block < 128 ? r->block : 128, false, 0, t->cfg);
    if (st != TP_OK) {
        delete t;
        return st;
    }
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = tape_alloc(t, &t->d_ckpt, (size_t)A.S * kAdjCkWords * (size_t)n * sizeof(float));
        if (e == cudaSuccess) e = tape_alloc(t, &t->d_u0, (size_t)n * 6 * sizeof(double));
    }
    if (e == cudaSuccess) e = tape_alloc(t, &t->d_gparam, 6 * sizeof(double));
    if (e == cudaSuccess) e = tape_alloc(t, &t->d_need, sizeof(int32_t));
    if (e != cudaSuccess) {
        delete t;
        return cuda_fail(ctx, e, "adjoint tape");
    }
    A.ckpt = t->d_ckpt;
    A.a.u0 = t->d_u0;
    A.g_param = t->d_gparam;
    *out = t;
    return TP_OK;
}

int adjoint_forward_on(tp_tape* t, const double* u0_dev, double* ufinal_dev, cudaStream_t s) {
    tp_ctx* ctx = t->ctx;
    AdjArgs& A = t->A;
    if (A.a.n == 0) return TP_OK;
    cudaError_t e = cudaMemcpyAsync(t->d_u0, u0_dev, (size_t)A.a.n * 6 * sizeof(double), cudaMemcpyDefault, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint initial states");
    A.u_final = ufinal_dev;
    e = launch_adjoint_forward(A, t->fk, t->cfg, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint forward launch");
    return TP_OK;
}

int adjoint_backward_on(tp_tape* t, const double* gfinal_dev, double* gu0_dev, double* gE_dev, double* gB_dev,
                        double* gparam_dev, cudaStream_t s) {
    tp_ctx* ctx = t->ctx;
    AdjArgs& A = t->A;
    if (t->E->id != t->E_id || t->B->id != t->B_id)
        return fail(ctx, TP_E_ARG, "a field was updated after the tape was recorded (rerun the tape)");
    const int64_t n = A.a.n;
    cudaError_t e = cudaSuccess;
    // segment records and node-gradient tables: allocated on first use, kept
    const int64_t rw = adjoint_record_words(t->fk, A.K, n);
    if (!t->d_rec && rw > 0) e = tape_alloc(t, &t->d_rec, (size_t)rw * sizeof(float));
    const int64_t sw = adjoint_state_words(t->fk, A.K, n);
    if (e == cudaSuccess && sw > 0 && !t->d_lam) e = tape_alloc(t, &t->d_lam, (size_t)sw * sizeof(float));
    const bool eb = t->fk == FK_EBGRID;
    const bool gridE = !eb && t->E->desc.kind == TP_FIELD_GRID;
    const bool gridB = !eb && t->B->desc.kind == TP_FIELD_GRID;
    if (e == cudaSuccess && eb && !t->d_geb) e = tape_alloc(t, &t->d_geb, (size_t)t->nodes_B * 2 * sizeof(float4));
    if (e == cudaSuccess && gridE && !t->d_gE) e = tape_alloc(t, &t->d_gE, (size_t)t->nodes_E * sizeof(float4));
    if (e == cudaSuccess && gridB && !t->d_gB) e = tape_alloc(t, &t->d_gB, (size_t)t->nodes_B * sizeof(float4));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint scratch");
    A.rec = t->d_rec;
    A.lam = t->d_lam;
    A.g_eb = t->d_geb;
    A.g_E = t->d_gE;
    A.g_B = t->d_gB;
    A.g_final = gfinal_dev;
    A.g_u0 = gu0_dev;
    A.need = t->d_need;
    // A pass whose node contributions reached 2^(G+100) could overflow the
    // float32 tables (and one far below 2^(G-100) loses their low bits): it
    // is repeated with G moved to the needed exponent minus 90.  The chosen
    // G is kept, so repeated passes of one problem run once.
    for (int attempt = 0; attempt < 3; ++attempt) {
        A.G = t->G;
        if (eb) e = cudaMemsetAsync(t->d_geb, 0, (size_t)t->nodes_B * 2 * sizeof(float4), s);
        if (e == cudaSuccess && gridE) e = cudaMemsetAsync(t->d_gE, 0, (size_t)t->nodes_E * sizeof(float4), s);
        if (e == cudaSuccess && gridB) e = cudaMemsetAsync(t->d_gB, 0, (size_t)t->nodes_B * sizeof(float4), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(t->d_gparam, 0, 6 * sizeof(double), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(t->d_need, 0x80, sizeof(int32_t), s);  // very negative
        if (e == cudaSuccess && n > 0) e = launch_adjoint_backward(A, t->fk, t->cfg, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint backward launch");
        if (!eb && !gridE && !gridB) break;  // no tables
        int32_t need = 0;
        e = cudaMemcpyAsync(&need, t->d_need, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint backward");
        if (need < -(1 << 30)) break;  // no node contribution at all
        if (need - t->G <= 100 && need - t->G >= -100) break;
        t->G = need - 90;
        if (attempt == 2) return fail(ctx, TP_E_OVERFLOW, "node-gradient range could not be fitted");
    }
    const int G = t->G;
    // grid parameter (uniform offset) gradients are the node-gradient sums
    if (eb) {
        e = launch_table_sum(t->d_geb, t->nodes_B, 2, 0, G, t->d_gparam, s);
        if (e == cudaSuccess) e = launch_table_sum(t->d_geb, t->nodes_B, 2, 1, G, t->d_gparam + 3, s);
        if (e == cudaSuccess && gE_dev) e = launch_table_unpack(t->d_geb, t->nodes_B, 2, 0, G, gE_dev, s);
        if (e == cudaSuccess && gB_dev) e = launch_table_unpack(t->d_geb, t->nodes_B, 2, 1, G, gB_dev, s);
    }
    if (e == cudaSuccess && gridE) {
        e = launch_table_sum(t->d_gE, t->nodes_E, 1, 0, G, t->d_gparam, s);
        if (e == cudaSuccess && gE_dev) e = launch_table_unpack(t->d_gE, t->nodes_E, 1, 0, G, gE_dev, s);
    }
    if (e == cudaSuccess && gridB) {
        e = launch_table_sum(t->d_gB, t->nodes_B, 1, 0, G, t->d_gparam + 3, s);
        if (e == cudaSuccess && gB_dev) e = launch_table_unpack(t->d_gB, t->nodes_B, 1, 0, G, gB_dev, s);
    }
    if (e == cudaSuccess && gparam_dev)
        e = cudaMemcpyAsync(gparam_dev, t->d_gparam, 6 * sizeof(double), cudaMemcpyDefault, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint gradient reduction");
    return TP_OK;
}

}  // namespace

extern "C" {

int tp_adjoint_forward_device(tp_ctx* ctx, const tp_adj_desc* d, const tp_field* E, const tp_field* B,
                              const double* u0, int64_t n, double* u_final, tp_tape** tape, void* stream) {
    if (!tape) return fail(ctx, TP_E_ARG, "null tape pointer");
    *tape = nullptr;
    if (n > 0 && (!u0 || !u_final)) return fail(ctx, TP_E_ARG, "null state buffer");
    tp_tape* t = nullptr;
    int st = adjoint_prepare(ctx, d, E, B, n, &t);
    if (st != TP_OK) return st;
    DeviceGuard g(ctx->device);
    st = adjoint_forward_on(t, u0, u_final, (cudaStream_t)stream);
    if (st != TP_OK) {
        delete t;
        return st;
    }
    *tape = t;
    return TP_OK;
}

int tp_adjoint_backward_device(tp_tape* t, const double* grad_final, double* grad_u0, double* grad_E,
                               double* grad_B, double* grad_param, void* stream) {
    if (!t) return TP_E_ARG;
    if (t->A.a.n > 0 && (!grad_final || !grad_u0)) return fail(t->ctx, TP_E_ARG, "null gradient buffer");
    DeviceGuard g(t->ctx->device);
    return adjoint_backward_on(t, grad_final, grad_u0, grad_E, grad_B, grad_param, (cudaStream_t)stream);
}

int tp_adjoint_forward(tp_ctx* ctx, const tp_adj_desc* d, const tp_field* E, const tp_field* B,
                       const double* u0, int64_t n, double* u_final, tp_tape** tape) {
    if (!tape) return fail(ctx, TP_E_ARG, "null tape pointer");
    *tape = nullptr;
    if (n > 0 && (!u0 || !u_final)) return fail(ctx, TP_E_ARG, "null state buffer");
    tp_tape* t = nullptr;
    int st = adjoint_prepare(ctx, d, E, B, n, &t);
    if (st != TP_OK) return st;
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    DBuf uf;
    cudaError_t e = uf.alloc((size_t)n * 6 * sizeof(double));
    if (e != cudaSuccess) {
        delete t;
        return cuda_fail(ctx, e, "adjoint final states");
    }
    st = adjoint_forward_on(t, u0, uf.as<double>(), ctx->stream);
    if (st == TP_OK && n > 0) {
        e = cudaMemcpyAsync(u_final, uf.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "adjoint forward");
    }
    if (st != TP_OK) {
        delete t;
        return st;
    }
    *tape = t;
    return TP_OK;
}

int tp_adjoint_backward(tp_tape* t, const double* grad_final, double* grad_u0, double* grad_E, double* grad_B,
                        double* grad_param) {
    if (!t) return TP_E_ARG;
    tp_ctx* ctx = t->ctx;
    const int64_t n = t->A.a.n;
    if (n > 0 && (!grad_final || !grad_u0)) return fail(ctx, TP_E_ARG, "null gradient buffer");
    DeviceGuard g(ctx->device);
    AllocStream alloc_stream(ctx->stream);
    const bool eb = t->fk == FK_EBGRID;
    const int64_t nE = (eb || t->E->desc.kind == TP_FIELD_GRID) ? t->nodes_E : 0;
    const int64_t nB = (eb || t->B->desc.kind == TP_FIELD_GRID) ? t->nodes_B : 0;
    DBuf gf, gu, ge, gb, gp;
    cudaError_t e = gf.alloc((size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess) e = gu.alloc((size_t)n * 6 * sizeof(double));
    if (e == cudaSuccess && grad_E && nE) e = ge.alloc((size_t)nE * 3 * sizeof(double));
    if (e == cudaSuccess && grad_B && nB) e = gb.alloc((size_t)nB * 3 * sizeof(double));
    if (e == cudaSuccess) e = gp.alloc(6 * sizeof(double));
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpyAsync(gf.p, grad_final, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint buffers");
    int st = adjoint_backward_on(t, gf.as<double>(), gu.as<double>(), ge.as<double>(), gb.as<double>(),
                                 gp.as<double>(), ctx->stream);
    if (st != TP_OK) return st;
    if (n > 0) e = cudaMemcpyAsync(grad_u0, gu.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && ge.p)
        e = cudaMemcpyAsync(grad_E, ge.p, (size_t)nE * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && gb.p)
        e = cudaMemcpyAsync(grad_B, gb.p, (size_t)nB * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && grad_param)
        e = cudaMemcpyAsync(grad_param, gp.p, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint backward");
    return TP_OK;
}

int tp_tape_rerun_device(tp_tape* t, const double* u0, double* u_final, void* stream) {
    if (!t) return TP_E_ARG;
    tp_ctx* ctx = t->ctx;
    if (t->A.a.n > 0 && (!u0 || !u_final)) return fail(ctx, TP_E_ARG, "null state buffer");
    DeviceGuard g(ctx->device);
    // refresh the field tables: a field may have been updated since the recording
    DevFields f;
    int st = make_dev_fields(ctx, t->E, const_cast<tp_field*>(t->B), f);
    if (st != TP_OK) return st;
    t->A.a.f = f;
    t->E_id = t->E->id;
    t->B_id = t->B->id;
    return adjoint_forward_on(t, u0, u_final, (cudaStream_t)stream);
}

int tp_tape_info(const tp_tape* t, int64_t* device_bytes, int64_t* nsteps) {
    if (!t) return TP_E_ARG;
    if (device_bytes) *device_bytes = t->bytes;
    if (nsteps) *nsteps = t->A.nt;
    return TP_OK;
}

int tp_tape_segments(const tp_tape* t, int64_t* checkpoint_every, int64_t* segments) {
    if (!t) return TP_E_ARG;
    if (checkpoint_every) *checkpoint_every = t->A.K;
    if (segments) *segments = t->A.S;
    return TP_OK;
}

void tp_tape_destroy(tp_tape* t) {
    if (!t) return;
    DeviceGuard g(t->ctx->device);
    cudaStreamSynchronize(t->ctx->stream);
    cudaDeviceSynchronize();
    delete t;
}

}  // extern "C"

namespace tpb {
int ctx_device(const tp_ctx* ctx) { return ctx->device; }
int ctx_fail(tp_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}
}  // namespace tpb
