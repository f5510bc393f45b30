// Request server for FISTA-CS slices (continuous batching on one device).
//
// Each admitted request runs its own chain -- upload, row IDFT, fused column
// FISTA (or the 2-D engine), RSS, download -- on one stream of a pool, so
// requests that arrive while others are running overlap with them on the
// GPU.  Admission is by an HBM budget and an in-flight limit: a request that
// does not fit is refused with OKS_EAGAIN and may be resubmitted once others
// complete.  Device memory per request comes from the stream-ordered pool
// (cudaMallocAsync) and is returned stream-ordered when the chain ends.
// All entry points are serialised by one mutex, so any host thread may call
// them; waits are bounded by the caller's timeout.
#include <chrono>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "ctx.h"

struct okscuda_server {
    okscuda_ctx* ctx = nullptr;
    std::mutex mu;
    std::vector<cudaStream_t> streams;
    int next_stream = 0;
    int max_inflight = 32;
    size_t budget = 0;
    size_t reserved = 0;
    uint64_t next_id = 1;
    struct Req {
        cudaEvent_t done = nullptr;
        size_t bytes = 0;
        int status = OKS_OK;
        bool finished = false;
        // pageable output: the device result goes to a pinned bounce buffer
        // and is copied to the caller's buffer when completion is observed
        void* bounce = nullptr;
        size_t bounce_bytes = 0;
        void* user_out = nullptr;
    };
    std::unordered_map<uint64_t, Req> reqs;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<void*, size_t>> pinned_pool;   // free pinned bounce buffers
    long long completed = 0;
};

namespace {

// Marks finished requests and returns their reservations (mutex held).
void reap(okscuda_server* s) {
    for (auto& kv : s->reqs) {
        auto& r = kv.second;
        if (r.finished) continue;
        const cudaError_t q = cudaEventQuery(r.done);
        if (q == cudaErrorNotReady) continue;
        r.finished = true;
        if (q != cudaSuccess) r.status = OKS_ECUDA;
        if (r.bounce) {
            if (r.status == OKS_OK) std::memcpy(r.user_out, r.bounce, r.bounce_bytes);
            s->pinned_pool.push_back({r.bounce, r.bounce_bytes});
            r.bounce = nullptr;
        }
        s->reserved -= r.bytes;
        s->completed += 1;
    }
}

// A pinned buffer of at least `bytes` from the pool (or a new one).
void* take_pinned(okscuda_server* s, size_t bytes, size_t* got) {
    for (size_t i = 0; i < s->pinned_pool.size(); ++i)
        if (s->pinned_pool[i].second >= bytes) {
            auto b = s->pinned_pool[i];
            s->pinned_pool.erase(s->pinned_pool.begin() + i);
            *got = b.second;
            return b.first;
        }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    *got = bytes;
    return p;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

cudaEvent_t take_event(okscuda_server* s) {
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
}

}  // namespace

extern "C" {

int okscuda_server_create(okscuda_ctx* ctx, const okscuda_server_cfg* cfg, okscuda_server** out) {
    OKS_CHECK_CTX();
    if (!out) return set_err(ctx, OKS_EINVAL, "server_create: null out");
    *out = nullptr;
    auto* s = new okscuda_server();
    s->ctx = ctx;
    const int ns = (cfg && cfg->n_streams > 0) ? cfg->n_streams : 8;
    s->max_inflight = (cfg && cfg->max_inflight > 0) ? cfg->max_inflight : 32;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = (cfg && cfg->hbm_budget_bytes > 0) ? cfg->hbm_budget_bytes : free_b / 2;
    for (int i = 0; i < ns; ++i) {
        cudaStream_t st;
        cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            for (auto x : s->streams) cudaStreamDestroy(x);
            delete s;
            return cuda_err(ctx, e, "server streams");
        }
        s->streams.push_back(st);
    }
    // keep freed pool memory for reuse between requests
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = s;
    return OKS_OK;
}

void okscuda_server_destroy(okscuda_server* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    for (auto st : s->streams) cudaStreamSynchronize(st);
    for (auto& kv : s->reqs) {
        cudaEventDestroy(kv.second.done);
        if (kv.second.bounce) cudaFreeHost(kv.second.bounce);
    }
    for (auto& b : s->pinned_pool) cudaFreeHost(b.first);
    for (auto e : s->ev_pool) cudaEventDestroy(e);
    for (auto st : s->streams) cudaStreamDestroy(st);
    delete s;
}

int okscuda_server_submit(okscuda_server* s, const okscuda_request* q, uint64_t* id) {
    if (!s || !q || !id) return OKS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    okscuda_ctx* ctx = s->ctx;
    OKS_CHECK_CTX();
    if ((!q->h_kspace && !q->d_kspace) || !q->h_mask || !q->h_rss || q->nc <= 0 || q->ny <= 0 || q->nx <= 0 ||
        q->iters < 0)
        return set_err(ctx, OKS_EINVAL, "server_submit: bad request");
    if (q->ny % 2 || q->nx % 2)
        return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", q->ny, q->nx);
    reap(s);
    const size_t N = (size_t)q->ny * q->nx;
    const size_t kbytes = sizeof(float2) * (size_t)q->nc * N;
    // k-space (solved in place) + RSS + the 2-D engine's worst-case scratch
    const size_t need = kbytes + sizeof(float) * N + 3 * kbytes;
    int inflight = 0;
    for (auto& kv : s->reqs) inflight += kv.second.finished ? 0 : 1;
    if (inflight >= s->max_inflight || s->reserved + need > s->budget)
        return set_err(ctx, OKS_EAGAIN, "admission refused: %d in flight, %zu of %zu bytes reserved", inflight,
                       s->reserved, s->budget);
    cudaStream_t st = s->streams[s->next_stream];
    s->next_stream = (s->next_stream + 1) % (int)s->streams.size();
    cudaStream_t saved = ctx->stream;
    ctx->stream = st;   // the request's chain runs on its own stream
    int rc = OKS_OK;
    void* dk = nullptr;
    void* drss = nullptr;
    cudaError_t e = cudaSuccess;
    if (q->h_kspace) {
        e = cudaMallocAsync(&dk, kbytes, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dk, q->h_kspace, kbytes, cudaMemcpyHostToDevice, st);
    } else {
        dk = const_cast<okscuda_c64*>(q->d_kspace);
    }
    if (e == cudaSuccess) e = cudaMallocAsync(&drss, sizeof(float) * N, st);
    if (e != cudaSuccess) rc = cuda_err(ctx, e, "server_submit: device memory");
    void* coils = nullptr;
    if (!rc && !q->h_kspace) {
        // device-resident input is left untouched: solve into a copy
        e = cudaMallocAsync(&coils, kbytes, st);
        if (e != cudaSuccess) rc = cuda_err(ctx, e, "server_submit: coil buffer");
    }
    okscuda_c64* work = static_cast<okscuda_c64*>(coils ? coils : dk);
    if (!rc) rc = oks_fista_core(ctx, static_cast<const okscuda_c64*>(dk), q->h_mask, 1, q->nc, q->ny, q->nx,
                                 q->iters, q->lambda, work);
    if (!rc) rc = okscuda_rss_crop(ctx, work, q->nc, q->ny, q->nx, q->ny, q->nx, static_cast<float*>(drss));
    void* bounce = nullptr;
    size_t bounce_cap = 0;
    if (!rc) {
        // a copy into pageable memory would block this call until the chain
        // ends; bounce through pinned memory instead
        void* dst = q->h_rss;
        if (!is_pinned(q->h_rss)) {
            bounce = take_pinned(s, sizeof(float) * N, &bounce_cap);
            if (!bounce) rc = set_err(ctx, OKS_ENOMEM, "server_submit: pinned bounce buffer");
            dst = bounce;
        }
        if (!rc) e = cudaMemcpyAsync(dst, drss, sizeof(float) * N, cudaMemcpyDeviceToHost, st);
        if (!rc && e != cudaSuccess) rc = cuda_err(ctx, e, "server_submit: download");
    }
    if (q->h_kspace && dk) cudaFreeAsync(dk, st);
    if (coils) cudaFreeAsync(coils, st);
    if (drss) cudaFreeAsync(drss, st);
    okscuda_server::Req r;
    r.done = take_event(s);
    cudaEventRecord(r.done, st);
    ctx->stream = saved;
    if (rc) {
        cudaEventSynchronize(r.done);
        if (bounce) s->pinned_pool.push_back({bounce, bounce_cap});
        s->ev_pool.push_back(r.done);
        return rc;
    }
    r.bounce = bounce;
    r.bounce_bytes = sizeof(float) * N;
    r.user_out = q->h_rss;
    r.bytes = need;
    s->reserved += need;
    *id = s->next_id++;
    s->reqs[*id] = r;
    return OKS_OK;
}

int okscuda_server_poll(okscuda_server* s, uint64_t id, int* done) {
    if (!s || !done) return OKS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    cudaSetDevice(s->ctx->device);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_err(s->ctx, OKS_EINVAL, "unknown request %llu", (unsigned long long)id);
    reap(s);
    *done = it->second.finished ? 1 : 0;
    if (it->second.finished) {
        const int st = it->second.status;
        s->ev_pool.push_back(it->second.done);
        s->reqs.erase(it);
        return st;
    }
    return OKS_OK;
}

int okscuda_server_wait(okscuda_server* s, uint64_t id, int timeout_ms) {
    if (!s) return OKS_EINVAL;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        int done = 0;
        const int rc = okscuda_server_poll(s, id, &done);
        if (rc != OKS_OK || done) return rc;
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
        if (timeout_ms >= 0 && ms.count() >= timeout_ms)
            return set_err(s->ctx, OKS_ETIMEDOUT, "request %llu not done after %d ms", (unsigned long long)id,
                           timeout_ms);
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int okscuda_server_stats(okscuda_server* s, long long* inflight, long long* completed, size_t* reserved_bytes) {
    if (!s) return OKS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    cudaSetDevice(s->ctx->device);
    reap(s);
    long long n = 0;
    for (auto& kv : s->reqs) n += kv.second.finished ? 0 : 1;
    if (inflight) *inflight = n;
    if (completed) *completed = s->completed;
    if (reserved_bytes) *reserved_bytes = s->reserved;
    return OKS_OK;
}

}  // extern "C"
