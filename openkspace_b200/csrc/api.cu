// C-ABI of the FISTA-CS path (include/okscuda.h): contexts, device memory,
// FFT plans and the dispatch of the sm_100a kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/okscuda.h"
#include "kernels.h"
#include "plan.h"

using oks::DevPlan;

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
};

namespace {

int set_err(okscuda_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_err(okscuda_ctx* c, cudaError_t e, const char* where) {
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

int ensure_scratch(okscuda_ctx* ctx, size_t bytes) {
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
int get_alpha(okscuda_ctx* ctx, int iters, const float** out) {
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

int get_plan(okscuda_ctx* ctx, int n, const DevPlan** out) {
    std::string msg;
    const DevPlan* p = ctx->plans.get(n, &msg);
    if (!p) return set_err(ctx, OKS_ECUDA, "FFT plan for n=%d: %s", n, msg.c_str());
    *out = p;
    return OKS_OK;
}

// Row mask of a 2-D mask when every row is all-0 or all-1.
bool separable_rows(const uint8_t* mask, int ny, int nx, std::vector<uint8_t>* rows) {
    rows->assign(ny, 0);
    for (int r = 0; r < ny; ++r) {
        const uint8_t* m = mask + (size_t)r * nx;
        const bool on = m[0] != 0;
        for (int x = 1; x < nx; ++x)
            if ((m[x] != 0) != on) return false;
        (*rows)[r] = on ? 1 : 0;
    }
    return true;
}

}  // namespace

// ====================================================================== C-ABI
extern "C" {

const char* okscuda_version(void) { return "okscuda 0.1 (sm_100a)"; }

int okscuda_create(int device, okscuda_ctx** out) {
    if (!out) return OKS_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return OKS_ECUDA;
    if (device < 0 || device >= ndev) return OKS_EINVAL;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return OKS_ECUDA;
    auto* c = new okscuda_ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return OKS_ECUDA; }
    c->stream = c->own_stream;
    *out = c;
    return OKS_OK;
}

void okscuda_destroy(okscuda_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->alpha) cudaFree(kv.second);
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->plans.clear();
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

int okscuda_last_error(const okscuda_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || len == 0) return OKS_EINVAL;
    std::snprintf(buf, len, "%s", ctx->err.c_str());
    return OKS_OK;
}

int okscuda_set_stream(okscuda_ctx* ctx, void* stream) {
    if (!ctx) return OKS_EINVAL;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return OKS_OK;
}

void* okscuda_get_stream(okscuda_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int okscuda_synchronize(okscuda_ctx* ctx) {
    OKS_CHECK_CTX();
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    return OKS_OK;
}

int okscuda_malloc(okscuda_ctx* ctx, size_t bytes, void** d_ptr) {
    OKS_CHECK_CTX();
    if (!d_ptr) return set_err(ctx, OKS_EINVAL, "okscuda_malloc: null out pointer");
    *d_ptr = nullptr;
    if (bytes == 0) return OKS_OK;
    OKS_CUDA(cudaMalloc(d_ptr, bytes));
    return OKS_OK;
}

int okscuda_free(okscuda_ctx* ctx, void* d_ptr) {
    OKS_CHECK_CTX();
    if (!d_ptr) return OKS_OK;
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    OKS_CUDA(cudaFree(d_ptr));
    return OKS_OK;
}

int okscuda_upload(okscuda_ctx* ctx, void* d_dst, const void* h_src, size_t bytes) {
    OKS_CHECK_CTX();
    if (bytes == 0) return OKS_OK;
    if (!d_dst || !h_src) return set_err(ctx, OKS_EINVAL, "okscuda_upload: null pointer");
    OKS_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return OKS_OK;
}

int okscuda_download(okscuda_ctx* ctx, void* h_dst, const void* d_src, size_t bytes) {
    OKS_CHECK_CTX();
    if (bytes == 0) return OKS_OK;
    if (!h_dst || !d_src) return set_err(ctx, OKS_EINVAL, "okscuda_download: null pointer");
    OKS_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    return OKS_OK;
}

int okscuda_host_alloc(okscuda_ctx* ctx, size_t bytes, void** h_ptr) {
    OKS_CHECK_CTX();
    if (!h_ptr) return OKS_EINVAL;
    OKS_CUDA(cudaMallocHost(h_ptr, bytes ? bytes : 1));
    return OKS_OK;
}

int okscuda_host_free(okscuda_ctx* ctx, void* h_ptr) {
    OKS_CHECK_CTX();
    if (h_ptr) OKS_CUDA(cudaFreeHost(h_ptr));
    return OKS_OK;
}

// ------------------------------------------------------------- primitives
int okscuda_centred_fft2(okscuda_ctx* ctx, okscuda_c64* d_data, int batch, int ny, int nx, int inverse) {
    OKS_CHECK_CTX();
    if (!d_data || batch < 0 || ny <= 0 || nx <= 0)
        return set_err(ctx, OKS_EINVAL, "okscuda_centred_fft2: bad arguments");
    if (batch == 0) return OKS_OK;
    const DevPlan *px, *py;
    int rc = get_plan(ctx, nx, &px);
    if (rc) return rc;
    rc = get_plan(ctx, ny, &py);
    if (rc) return rc;
    float2* d = reinterpret_cast<float2*>(d_data);
    oks::RowXformArgs ra{};
    ra.in = d; ra.out = d; ra.nrows = (long long)batch * ny; ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = inverse ? +1 : -1; ra.centred = 1; ra.scale = 1.0f; ra.rows_per_prob = ny;
    OKS_CUDA(oks::launch_row_xform(ra, oks::RowBits{}, *px, ctx->stream));
    oks::ColXformArgs ca{};
    ca.data = d; ca.nprob = batch; ca.ny = ny; ca.nx = nx; ca.prob_stride = (long long)ny * nx;
    ca.sign = inverse ? +1 : -1; ca.centred = 1;
    ca.scale = 1.0f / std::sqrt((float)ny * (float)nx);
    OKS_CUDA(oks::launch_col_xform(ca, *py, ctx->stream));
    return OKS_OK;
}

static int haar_common(okscuda_ctx* ctx, const okscuda_c64* in, okscuda_c64* out, int batch, int ny,
                       int nx, int inverse) {
    OKS_CHECK_CTX();
    if (!in || !out || batch < 0 || ny <= 0 || nx <= 0)
        return set_err(ctx, OKS_EINVAL, "haar: bad arguments");
    if (ny % 2 || nx % 2) return set_err(ctx, OKS_EODD, "Haar: dims must be even");
    if (in == out) return set_err(ctx, OKS_EINVAL, "haar: in and out must differ");
    OKS_CUDA(oks::launch_haar(reinterpret_cast<const float2*>(in), reinterpret_cast<float2*>(out), batch,
                              ny, nx, inverse, ctx->stream));
    return OKS_OK;
}

int okscuda_haar_forward(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, int batch, int ny,
                         int nx) {
    return haar_common(ctx, d_in, d_out, batch, ny, nx, 0);
}

int okscuda_haar_inverse(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, int batch, int ny,
                         int nx) {
    return haar_common(ctx, d_in, d_out, batch, ny, nx, 1);
}

int okscuda_soft_threshold_details(okscuda_ctx* ctx, okscuda_c64* d_data, int batch, int ny, int nx,
                                   float lambda) {
    OKS_CHECK_CTX();
    if (!d_data || batch < 0 || ny <= 0 || nx <= 0)
        return set_err(ctx, OKS_EINVAL, "soft_threshold: bad arguments");
    OKS_CUDA(oks::launch_soft_threshold(reinterpret_cast<float2*>(d_data), batch, ny, nx, lambda,
                                        ctx->stream));
    return OKS_OK;
}

int okscuda_rss_crop(okscuda_ctx* ctx, const okscuda_c64* d_coils, int nc, int ny, int nx, int ty, int tx,
                     float* d_out) {
    OKS_CHECK_CTX();
    if (!d_coils || !d_out || nc < 0 || ny <= 0 || nx <= 0 || ty <= 0 || tx <= 0 || ty > ny || tx > nx)
        return set_err(ctx, OKS_EINVAL, "rss_crop: bad arguments");
    oks::RssArgs a{};
    a.coils = reinterpret_cast<const float2*>(d_coils);
    a.coil_stride = (long long)ny * nx;
    a.nc = nc; a.ny = ny; a.nx = nx;
    a.ty = ty; a.tx = tx; a.y0 = (ny - ty) / 2; a.x0 = (nx - tx) / 2;
    a.out = d_out;
    OKS_CUDA(oks::launch_rss(a, ctx->stream));
    return OKS_OK;
}

// ---------------------------------------------------------------- FISTA-CS
static int fista_core(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int batch,
                      int ny, int nx, int iters, float lambda, okscuda_c64* d_out) {
    if (!d_kspace || !h_mask || !d_out || batch < 0 || ny <= 0 || nx <= 0 || iters < 0)
        return set_err(ctx, OKS_EINVAL, "fista_cs: bad arguments");
    if (ny % 2 || nx % 2)
        return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", ny, nx);
    if (batch == 0) return OKS_OK;
    std::vector<uint8_t> rows;
    if (!separable_rows(h_mask, ny, nx, &rows))
        return set_err(ctx, OKS_ENOTSUP, "fista_cs: mask varies along kx (general 2-D mask path not built)");
    const DevPlan *px, *py;
    int rc = get_plan(ctx, nx, &px);
    if (rc) return rc;
    rc = get_plan(ctx, ny, &py);
    if (rc) return rc;
    const float* alpha = nullptr;
    rc = get_alpha(ctx, iters, &alpha);
    if (rc) return rc;
    if (ny > oks::kMaxMaskRows)
        return set_err(ctx, OKS_ENOTSUP, "fista_cs: ny=%d above %d", ny, oks::kMaxMaskRows);
    oks::RowBits bits{};
    for (int r = 0; r < ny; ++r)
        if (rows[r]) bits.w[r >> 5] |= 1u << (r & 31);

    // y' = sqrt(ny) (-1)^{ny/2} (-1)^r * centred unitary row-IDFT of y
    float2* out = reinterpret_cast<float2*>(d_out);
    oks::RowXformArgs ra{};
    ra.in = reinterpret_cast<const float2*>(d_kspace);
    ra.out = out;
    ra.nrows = (long long)batch * ny;
    ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = +1; ra.centred = 1;
    ra.scale = std::sqrt((float)ny) / std::sqrt((float)nx) * (((ny / 2) & 1) ? -1.0f : 1.0f);
    ra.rows_per_prob = ny; ra.rowsign = 1;
    ra.use_keep = 1;
    OKS_CUDA(oks::launch_row_xform(ra, bits, *px, ctx->stream));

    oks::FistaColArgs fa{};
    fa.ytil = out; fa.prob_stride = (long long)ny * nx;
    fa.minv = 1.0f / (float)ny;
    fa.xout = out; fa.out_stride = (long long)ny * nx;
    fa.ny = ny; fa.nx = nx; fa.iters = iters; fa.lambda = lambda; fa.alpha = alpha;
    fa.nprob = batch;
    OKS_CUDA(oks::launch_fista_col(fa, bits, *py, ctx->stream));
    return OKS_OK;
}

int okscuda_fista_cs(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int batch, int ny,
                     int nx, int iters, float lambda, okscuda_c64* d_out) {
    OKS_CHECK_CTX();
    return fista_core(ctx, d_kspace, h_mask, batch, ny, nx, iters, lambda, d_out);
}

int okscuda_cs_slice(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc, int ny,
                     int nx, int iters, float lambda, float* d_rss, okscuda_c64* d_coils) {
    OKS_CHECK_CTX();
    if (!d_rss) return set_err(ctx, OKS_EINVAL, "cs_slice: null output");
    okscuda_c64* coils = d_coils;
    void* own = nullptr;
    if (!coils) {
        OKS_CUDA(cudaMallocAsync(&own, sizeof(okscuda_c64) * (size_t)nc * ny * nx, ctx->stream));
        coils = static_cast<okscuda_c64*>(own);
    }
    int rc = fista_core(ctx, d_kspace, h_mask, nc, ny, nx, iters, lambda, coils);
    if (rc == OKS_OK) rc = okscuda_rss_crop(ctx, coils, nc, ny, nx, ny, nx, d_rss);
    if (own) cudaFreeAsync(own, ctx->stream);
    return rc;
}

}  // extern "C"
