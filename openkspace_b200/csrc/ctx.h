// Private: the okscuda_ctx definition and helpers shared by the C-ABI
// translation units (api.cu, strategy.cu).  Not part of the public header.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/okscuda.h"
#include "kernels.h"
#include "plan.h"

using oks::DevPlan;

// Plan and launch-shape choices of the FISTA engines for one shape (set by
// okscuda_set_option globally, or per shape by okscuda_autotune).
struct TuneParams {
    int col_engine;
    int col_variant;
    int persist2d;
    int occ2d;
    int prefetch2d;
    int fista2d_streams;
    long long fista2d_chunk;
};

struct okscuda_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    oks::PlanCache plans;
    std::map<int, float*> alpha;          // iters -> device alpha table
    // scratch (grow-only)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    oks::Staging staging;
    long long fista2d_chunk = 0;          // problems per 2-D-mask chunk (0 = auto)
    int col_engine = 0;                   // ky-only masks: 0 auto, 1 generic smem, 2 register-resident
    int col_variant = -1;                 // register column engine plan variant (-1: per-length default)
    int persist2d = 1;                    // 2-D register passes: persistent grid
    int mask_bits = 1;                    // 2-D passes: separable masks read as row/column bits
    int occ2d = 1;                        // 2-D register passes: launch bounds for 12 (1) or 18 (2) warps per SM
    int fista2d_streams = 2;              // 2-D engine: chunks in flight at once (forked streams)
    int prefetch2d = 1;                   // 2-D register column pass: pipelined loads (separable masks)
    // per-shape choices found by okscuda_autotune: key (kind, ny, nx), kind 0
    // = ky-only masks (column engine, nx = 0), kind 1 = 2-D masks
    std::map<std::tuple<int, int, int>, TuneParams> tuned;
    int use_tuned = 1;
    // 2-D engine CUDA graphs: key -> instantiated launch sequence over the
    // entry's own buffers (k-space in, coil images out, masks, scratch)
    struct Graph2d {
        cudaGraphExec_t exec = nullptr;
        void* y = nullptr;
        void* out = nullptr;
        void* masks = nullptr;
        void* scratch = nullptr;
        cudaEvent_t done = nullptr;
        bool failed = false;
        unsigned long long last_use = 0;
        long long kernels = 0;            // kernel nodes in the graph
    };
    std::map<std::string, Graph2d> g2d;
    unsigned long long g2d_clock = 0;
    int graph2d = 1;                      // 2-D engine: replay captured launch sequences
    oks::RegTables reg_tables;
    // tensor-core row DFT: split B operands per (n, sign, centred, column
    // sets), device column lists, error flag
    struct TcMat { void* hi = nullptr; void* lo = nullptr; int* in_cols = nullptr; int* out_cols = nullptr; };
    std::map<std::string, TcMat> tc_mats;
    int* tc_err = nullptr;                // [0] bounded-wait error word, [1] a word nothing sets (gate test)
    long long tc_gate_cycles = 0;         // > 0: tensor-core launches first wait on tc_err[1] (tests only)
    int row_engine = 0;                   // 2-D engine row pass: 0 SIMT FFT, 1 tensor-core DFT
    int xform_reg = 1;                    // row/column transforms: 1 register kernels where a plan exists
    int xform_tile = 0;                   // column pairs per CTA of the register column transform (0: by length)
    int xform_lanes = 0;                  // lanes-across-columns form of it: 0 by length, 1..4, -1 off
    int xform_lanes_pf = 1;               // lanes form: 1 = next tile staged in shared memory while transforming
    int xform_row_variant = 0;            // register row transform: alternative plans for 192 and 320
    int col2d_lanes = 0;                  // 2-D engine column pass: 0 by length, -1 column pairs, 1-12 a lanes form
    int pdl2d = 0;                        // 2-D register passes: programmatic dependent launches
    int row2d_ctas = 0;                   // 2-D row pass: CTAs per SM cap (0: every resident slot)
    int col2d_ctas = 0;                   // pruned 368 column pass: CTAs per SM cap (0: every resident slot)
    int prewhiten_bulk = -1;              // prewhitening: -1 by channel count, 1 bulk-copy staged kernel, 0 plain loads
    struct Aux { cudaStream_t stream = nullptr; cudaEvent_t done = nullptr; };
    std::vector<Aux> aux;                 // fork/join streams (okscuda_cs_batch)
    // host scratch kept across calls (no page faults on every call): the 2-D
    // engine's mask upload image and the placement's filled mask
    std::vector<uint8_t> h_mask_up, h_filled;
    cudaEvent_t fork_ev = nullptr;
    // per-launch CUDA-event profiling (okscuda_profile_*)
    bool prof_on = false;
    // kernels = kernel launches inside the bracket (the node count of a replayed graph)
    struct ProfRec { const char* name; cudaEvent_t a, b; long long kernels; };
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
};

namespace oks_internal {

inline int set_err(okscuda_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

inline int cuda_err(okscuda_ctx* c, cudaError_t e, const char* where) {
    return set_err(c, e == cudaErrorMemoryAllocation ? OKS_ENOMEM : OKS_ECUDA, "%s: %s (%s)", where,
                   cudaGetErrorString(e), cudaGetErrorName(e));
}

#define OKS_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_err(ctx, e_, #call); \
    } while (0)

#define OKS_CHECK_CTX()                                                  \
    do {                                                                 \
        if (!ctx) return OKS_EINVAL;                                     \
        cudaError_t e0_ = cudaSetDevice(ctx->device);                    \
        if (e0_ != cudaSuccess) return cuda_err(ctx, e0_, "cudaSetDevice"); \
    } while (0)

inline void free_graph2d(okscuda_ctx::Graph2d& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    cudaFree(g.y);
    cudaFree(g.out);
    cudaFree(g.masks);
    cudaFree(g.scratch);
    if (g.done) cudaEventDestroy(g.done);
    g.exec = nullptr;
    g.y = g.out = g.masks = g.scratch = nullptr;
    g.done = nullptr;
}

// The choices in force for a shape: the autotuned entry when there is one
// (and lookups are on), else the context-wide options.
inline TuneParams tune_params(const okscuda_ctx* ctx, int kind, int ny, int nx) {
    if (ctx->use_tuned) {
        auto it = ctx->tuned.find(std::make_tuple(kind, ny, kind == 0 ? 0 : nx));
        if (it != ctx->tuned.end()) return it->second;
    }
    // built-in plan variants, from okscuda_autotune runs and batched timings on
    // B200: the E = 8 alternative plan is faster for column lengths 256, 320,
    // 384 and 512
    const int variant =
        ctx->col_variant >= 0 ? ctx->col_variant : (ny == 256 || ny == 320 || ny == 384 || ny == 512) ? 1 : 0;
    return TuneParams{ctx->col_engine, variant, ctx->persist2d, ctx->occ2d,
                      ctx->prefetch2d, ctx->fista2d_streams, ctx->fista2d_chunk};
}

inline int ensure_scratch(okscuda_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->scratch_bytes) return OKS_OK;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
    if (e != cudaSuccess) return cuda_err(ctx, e, "cudaMalloc(scratch)");
    ctx->scratch_bytes = bytes;
    return OKS_OK;
}

// cs.rs:125-126 in f32, as the reference computes it.
inline int get_alpha(okscuda_ctx* ctx, int iters, const float** out) {
    auto it = ctx->alpha.find(iters);
    if (it != ctx->alpha.end()) { *out = it->second; return OKS_OK; }
    std::vector<float> h(iters > 0 ? iters : 1, 0.f);
    float t = 1.0f;
    for (int i = 0; i < iters; ++i) {
        float t_new = 0.5f * (1.0f + std::sqrt(1.0f + 4.0f * t * t));
        h[i] = (t - 1.0f) / t_new;
        t = t_new;
    }
    float* d = nullptr;
    OKS_CUDA(cudaMalloc(&d, sizeof(float) * h.size()));
    OKS_CUDA(cudaMemcpy(d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
    ctx->alpha[iters] = d;
    *out = d;
    return OKS_OK;
}

inline int get_plan(okscuda_ctx* ctx, int n, const DevPlan** out) {
    std::string msg;
    const DevPlan* p = ctx->plans.get(n, &msg);
    if (!p) return set_err(ctx, OKS_ECUDA, "FFT plan for n=%d: %s", n, msg.c_str());
    *out = p;
    return OKS_OK;
}

// Small host->device uploads (masks, tables) through a ring of pinned slots:
// the copy is enqueued on the context stream, and a slot is reused only after
// the event recorded behind the kernels that read it has completed.
inline int stage_upload(okscuda_ctx* ctx, const void* src, size_t bytes, oks::Staging::Slot** out) {
    oks::Staging::Slot* s;
    if (bytes >= oks::Staging::kBig) {
        s = &ctx->staging.big[ctx->staging.next_big];
        ctx->staging.next_big ^= 1;
    } else {
        s = &ctx->staging.slots[ctx->staging.next];
        ctx->staging.next = (ctx->staging.next + 1) % oks::Staging::kSlots;
    }
    if (s->ev) OKS_CUDA(cudaEventSynchronize(s->ev));
    else OKS_CUDA(cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming));
    if (bytes > s->cap) {
        if (s->host) cudaFreeHost(s->host);
        if (s->dev) cudaFree(s->dev);
        s->host = s->dev = nullptr;
        s->cap = 0;
        size_t cap = bytes < 4096 ? 4096 : bytes;
        OKS_CUDA(cudaMallocHost(&s->host, cap));
        OKS_CUDA(cudaMalloc(&s->dev, cap));
        s->cap = cap;
    }
    std::memcpy(s->host, src, bytes);
    OKS_CUDA(cudaMemcpyAsync(s->dev, s->host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    *out = s;
    return OKS_OK;
}

inline void stage_release(okscuda_ctx* ctx, oks::Staging::Slot* s) { cudaEventRecord(s->ev, ctx->stream); }

inline cudaEvent_t prof_event(okscuda_ctx* ctx) {
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Records CUDA events around one kernel launch (or one graph of `kernels`
// kernel launches) when profiling is on.
struct ProfScope {
    okscuda_ctx* ctx;
    cudaStream_t st;
    okscuda_ctx::ProfRec rec{};
    ProfScope(okscuda_ctx* c, const char* name, cudaStream_t s = nullptr, long long kernels = 1)
        : ctx(c), st(s ? s : c->stream) {
        if (!ctx->prof_on) return;
        rec.name = name;
        rec.kernels = kernels;
        rec.a = prof_event(ctx);
        rec.b = prof_event(ctx);
        cudaEventRecord(rec.a, st);
    }
    ~ProfScope() {
        if (!ctx->prof_on || !rec.a) return;
        cudaEventRecord(rec.b, st);
        ctx->prof.push_back(rec);
    }
};

// Auxiliary streams for fork/join inside one entry point.
inline int ensure_aux_streams(okscuda_ctx* ctx, int n) {
    if (!ctx->fork_ev) {
        cudaError_t e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_err(ctx, e, "fork event");
    }
    while ((int)ctx->aux.size() < n) {
        okscuda_ctx::Aux a;
        cudaError_t e = cudaStreamCreateWithFlags(&a.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a.done, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_err(ctx, e, "aux stream");
        ctx->aux.push_back(a);
    }
    return OKS_OK;
}

// Split (3xBF16) DFT matrix of length n from the columns in_idx to the
// columns out_idx (empty = all n), built once per context; the index lists
// are also kept on the device (nullptr when empty).
inline int tc_matrix(okscuda_ctx* ctx, int n, int sign, int centred, const std::vector<int>& in_idx,
                     const std::vector<int>& out_idx, const okscuda_ctx::TcMat** out) {
    std::string key = std::to_string(n) + "/" + std::to_string(sign) + "/" + std::to_string(centred) + "/i";
    for (int v : in_idx) key += std::to_string(v) + ",";
    key += "/o";
    for (int v : out_idx) key += std::to_string(v) + ",";
    auto it = ctx->tc_mats.find(key);
    if (it == ctx->tc_mats.end()) {
        std::vector<uint16_t> h, l;
        oks::tc::dft_matrix_split(n, sign, centred, in_idx, out_idx, &h, &l);
        okscuda_ctx::TcMat m;
        const size_t bytes = h.size() * sizeof(uint16_t);
        cudaError_t e = cudaMalloc(&m.hi, bytes);
        if (e == cudaSuccess) e = cudaMalloc(&m.lo, bytes);
        // pageable sources: each copy completes before cudaMemcpy returns
        if (e == cudaSuccess) e = cudaMemcpy(m.hi, h.data(), bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(m.lo, l.data(), bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !in_idx.empty()) {
            e = cudaMalloc(&m.in_cols, sizeof(int) * in_idx.size());
            if (e == cudaSuccess)
                e = cudaMemcpy(m.in_cols, in_idx.data(), sizeof(int) * in_idx.size(), cudaMemcpyHostToDevice);
        }
        if (e == cudaSuccess && !out_idx.empty()) {
            e = cudaMalloc(&m.out_cols, sizeof(int) * out_idx.size());
            if (e == cudaSuccess)
                e = cudaMemcpy(m.out_cols, out_idx.data(), sizeof(int) * out_idx.size(), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            cudaFree(m.hi);
            cudaFree(m.lo);
            cudaFree(m.in_cols);
            cudaFree(m.out_cols);
            return cuda_err(ctx, e, "tensor-core DFT matrix");
        }
        it = ctx->tc_mats.emplace(key, m).first;
    }
    *out = &it->second;
    return OKS_OK;
}

inline int tc_err_flag(okscuda_ctx* ctx) {
    if (!ctx->tc_err) {
        OKS_CUDA(cudaMalloc(&ctx->tc_err, 2 * sizeof(int)));
        OKS_CUDA(cudaMemset(ctx->tc_err, 0, 2 * sizeof(int)));
    }
    return OKS_OK;
}

}  // namespace oks_internal

using namespace oks_internal;

// FISTA on nprob problems [nprob][ny][nx] (problem b uses host mask b % nmask),
// dispatching to the fused column engine (ky-only masks) or the 2-D engine.
// okscuda_cs_batch on the context stream with the column-length groups on
// the fork streams aux[0..naux) (the context's own when aux is null).
int oks_cs_batch_core(okscuda_ctx* ctx, const okscuda_slice_req* reqs, int n, okscuda_ctx::Aux* aux, int naux,
                      cudaEvent_t fork_ev);
extern "C" int oks_fista_core(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nmask,
                              long long nprob, int ny, int nx, int iters, float lambda, okscuda_c64* d_out);
