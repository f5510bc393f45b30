// C-ABI of the FISTA-CS path (include/okscuda.h): contexts, device memory,
// FFT plans and the dispatch of the sm_100a kernels.
#include "ctx.h"

// ====================================================================== C-ABI
namespace oks {
// Readers of the per-translation-unit error words of the bounds-checked
// build (reg_fft.cuh registers one per unit at load; none in the normal build).
static std::vector<unsigned (*)(int)>& bounds_readers() {
    static std::vector<unsigned (*)(int)> v;
    return v;
}
void bounds_register(unsigned (*reader)(int clear)) { bounds_readers().push_back(reader); }
}  // namespace oks

extern "C" {

const char* okscuda_version(void) {
#ifdef OKS_BOUNDS_CHECK
    return "okscuda 0.1 (sm_100a, bounds-checked)";
#else
    return "okscuda 0.1 (sm_100a)";
#endif
}

int okscuda_debug_bounds(okscuda_ctx* ctx, unsigned int* word, int clear) {
    OKS_CHECK_CTX();
    if (!word) return set_err(ctx, OKS_EINVAL, "debug_bounds: null word");
    *word = 0;
#ifndef OKS_BOUNDS_CHECK
    (void)clear;
    return set_err(ctx, OKS_ENOTSUP, "debug_bounds: not a bounds-checked build (libokscuda_bounds.so)");
#else
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    OKS_CUDA(cudaDeviceSynchronize());
    for (auto r : oks::bounds_readers()) *word |= r(clear);
    return OKS_OK;
#endif
}

int okscuda_create(int device, okscuda_ctx** out) {
    if (!out) return OKS_EINVAL;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return OKS_ECUDA;
    if (device < 0 || device >= ndev) return OKS_EINVAL;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return OKS_ECUDA;
    // The engines take their scratch stream-ordered (cudaMallocAsync).  With
    // the pool's default release threshold of 0, every host synchronisation
    // returns that memory to the driver and the next call maps it again
    // (hundreds of ms for the GB-sized scratch of a volume); keep up to
    // 16 GiB cached in the device's default pool instead.
    {
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess && pool) {
            uint64_t keep = 16ull << 30, cur = 0;
            if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < keep)
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        (void)cudaGetLastError();
    }
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
    ctx->staging.release();
    for (auto& r : ctx->prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
    ctx->plans.clear();
    if (ctx->reg_tables.base) cudaFree(ctx->reg_tables.base);
    for (auto& kv : ctx->tc_mats) {
        cudaFree(kv.second.hi);
        cudaFree(kv.second.lo);
        cudaFree(kv.second.in_cols);
        cudaFree(kv.second.out_cols);
    }
    if (ctx->tc_err) cudaFree(ctx->tc_err);
    for (auto& kv : ctx->g2d) free_graph2d(kv.second);
    for (auto& a : ctx->aux) { cudaStreamDestroy(a.stream); cudaEventDestroy(a.done); }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

int okscuda_set_option(okscuda_ctx* ctx, const char* name, long long value) {
    if (!ctx || !name) return OKS_EINVAL;
    if (!std::strcmp(name, "col_engine")) {
        if (value < 0 || value > 2) return set_err(ctx, OKS_EINVAL, "col_engine: 0 auto, 1 generic, 2 register");
        ctx->col_engine = (int)value;
    } else if (!std::strcmp(name, "col_variant")) {
        if (value < -1 || value > 1) return set_err(ctx, OKS_EINVAL, "col_variant: -1 (per length), 0 or 1");
        ctx->col_variant = (int)value;
    } else if (!std::strcmp(name, "persist2d")) {
        ctx->persist2d = value != 0;
    } else if (!std::strcmp(name, "mask_bits")) {
        ctx->mask_bits = value != 0;
    } else if (!std::strcmp(name, "occ2d")) {
        if (value < 0 || value > 3)
            return set_err(ctx, OKS_EINVAL, "occ2d: 0 (1 CTA), 1 (12 warps), 2 (18 warps), 3 (15 warps)");
        ctx->occ2d = (int)value;
    } else if (!std::strcmp(name, "prefetch2d")) {
        if (value < 0 || value > 7)
            return set_err(ctx, OKS_EINVAL, "prefetch2d: bit 0 column pass, bit 1 row pass, bit 2 bulk-copy row pass");
        ctx->prefetch2d = (int)value;
    } else if (!std::strcmp(name, "graph2d")) {
        ctx->graph2d = value != 0;
        if (!ctx->graph2d) {
            cudaDeviceSynchronize();
            for (auto& kv : ctx->g2d) free_graph2d(kv.second);
            ctx->g2d.clear();
        }
    } else if (!std::strcmp(name, "autotune_use")) {
        ctx->use_tuned = value != 0;
    } else if (!std::strcmp(name, "autotune_clear")) {
        ctx->tuned.clear();
    } else if (!std::strcmp(name, "row_engine")) {
        if (value < 0 || value > 1) return set_err(ctx, OKS_EINVAL, "row_engine: 0 SIMT FFT, 1 tensor-core DFT");
        ctx->row_engine = (int)value;
    } else if (!std::strcmp(name, "xform_engine")) {
        if (value < 0 || value > 1) return set_err(ctx, OKS_EINVAL, "xform_engine: 0 shared-memory, 1 register");
        ctx->xform_reg = (int)value;
    } else if (!std::strcmp(name, "xform_tile")) {
        if (value != 0 && value != 2 && value != 4 && value != 8)
            return set_err(ctx, OKS_EINVAL, "xform_tile: 0 (by length), 2, 4 or 8 column pairs");
        ctx->xform_tile = (int)value;
    } else if (!std::strcmp(name, "col2d_lanes")) {
        if (value < -1 || value > 14)
            return set_err(ctx, OKS_EINVAL,
                           "col2d_lanes: -1 column pairs, 0 by length, 1 to 8 a lanes form, 9 to 14 the pruned 368 forms");
        ctx->col2d_lanes = (int)value;
    } else if (!std::strcmp(name, "xform_row_variant")) {
        if (value < 0 || value > 3) return set_err(ctx, OKS_EINVAL, "xform_row_variant: 0 to 3");
        ctx->xform_row_variant = (int)value;
    } else if (!std::strcmp(name, "pdl2d")) {
        if (value < 0 || value > 1) return set_err(ctx, OKS_EINVAL, "pdl2d: 0 or 1");
        ctx->pdl2d = (int)value;
    } else if (!std::strcmp(name, "row2d_ctas")) {
        if (value < 0 || value > 16) return set_err(ctx, OKS_EINVAL, "row2d_ctas: 0 to 16");
        ctx->row2d_ctas = (int)value;
    } else if (!std::strcmp(name, "col2d_ctas")) {
        if (value < 0 || value > 16) return set_err(ctx, OKS_EINVAL, "col2d_ctas: 0 to 16");
        ctx->col2d_ctas = (int)value;
    } else if (!std::strcmp(name, "prewhiten_bulk")) {
        if (value < -1 || value > 1) return set_err(ctx, OKS_EINVAL, "prewhiten_bulk: -1, 0 or 1");
        ctx->prewhiten_bulk = (int)value;
    } else if (!std::strcmp(name, "xform_lanes_pf")) {
        if (value < 0 || value > 1) return set_err(ctx, OKS_EINVAL, "xform_lanes_pf: 0 or 1");
        ctx->xform_lanes_pf = (int)value;
    } else if (!std::strcmp(name, "xform_lanes")) {
        if (value < -1 || value > 11) return set_err(ctx, OKS_EINVAL, "xform_lanes: -1 off, 0 by length, 1 to 11");
        ctx->xform_lanes = (int)value;
    } else if (!std::strcmp(name, "fista2d_streams")) {
        if (value < 1 || value > 8) return set_err(ctx, OKS_EINVAL, "fista2d_streams: 1 to 8");
        ctx->fista2d_streams = (int)value;
    } else if (!std::strcmp(name, "tc_gate_test")) {
        // tests of the bounded waits: the next tensor-core launches wait at
        // most `value` clock cycles on a device word nothing sets, then record
        // the time-out (code 7) and return without work; 0 turns it off
        if (value < 0) return set_err(ctx, OKS_EINVAL, "tc_gate_test must be >= 0");
        ctx->tc_gate_cycles = value;
    } else if (!std::strcmp(name, "fista2d_chunk")) {
        if (value < 0) return set_err(ctx, OKS_EINVAL, "fista2d_chunk must be >= 0");
        ctx->fista2d_chunk = value;
    } else {
        return set_err(ctx, OKS_EINVAL, "unknown option '%s'", name);
    }
    return OKS_OK;
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
    ra.reg = ctx->xform_reg;
    ra.variant = ctx->xform_row_variant;
    ra.in = d; ra.out = d; ra.nrows = (long long)batch * ny; ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = inverse ? +1 : -1; ra.centred = 1; ra.scale = 1.0f; ra.rows_per_prob = ny;
    {
        ProfScope ps(ctx, "k_row_xform");
        OKS_CUDA(oks::launch_row_xform(ra, *px, ctx->stream));
    }
    oks::ColXformArgs ca{};
    ca.reg = ctx->xform_reg; ca.tile = ctx->xform_tile; ca.lanes = ctx->xform_lanes; ca.lanes_pf = ctx->xform_lanes_pf;
    ca.data = d; ca.nprob = batch; ca.ny = ny; ca.nx = nx; ca.prob_stride = (long long)ny * nx;
    ca.sign = inverse ? +1 : -1; ca.centred = 1;
    ca.scale = 1.0f / std::sqrt((float)ny * (float)nx);
    ProfScope ps(ctx, "k_col_xform");
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
    ProfScope ps(ctx, "k_haar");
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
    ProfScope ps(ctx, "k_soft_threshold");
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
    a.nslice = 1; a.slice_stride = 0;
    a.ty = ty; a.tx = tx; a.y0 = (ny - ty) / 2; a.x0 = (nx - tx) / 2;
    a.out = d_out;
    ProfScope ps(ctx, "k_rss");
    OKS_CUDA(oks::launch_rss(a, ctx->stream));
    return OKS_OK;
}

// ---------------------------------------------------------------- FISTA-CS
// Row masks of `nmask` 2-D masks [nmask][ny][nx] when every row of every mask
// is all-0 or all-1 (a ky-only mask), packed 32 rows per word.
static bool pack_row_masks(const uint8_t* h_mask, int nmask, int ny, int nx, std::vector<uint32_t>* words,
                           int* wstride) {
    *wstride = (ny + 31) / 32;
    words->assign((size_t)nmask * *wstride, 0u);
    for (int k = 0; k < nmask; ++k)
        for (int r = 0; r < ny; ++r) {
            const uint8_t* m = h_mask + ((size_t)k * ny + r) * nx;
            const bool on = m[0] != 0;
            for (int x = 1; x < nx; ++x)
                if ((m[x] != 0) != on) return false;
            if (on) (*words)[(size_t)k * *wstride + (r >> 5)] |= 1u << (r & 31);
        }
    return true;
}

// FISTA with an arbitrary 2-D mask (not constant along kx): two passes per
// iteration over state kept in device memory, problems processed in chunks
// sized so the chunk's state stays resident in L2.
static int fista2d_core(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nmask,
                        long long nprob, int ny, int nx, int iters, float lambda, okscuda_c64* d_out) {
    const DevPlan *px, *py;
    int rc = get_plan(ctx, nx, &px);
    if (rc) return rc;
    rc = get_plan(ctx, ny, &py);
    if (rc) return rc;
    const float* alpha = nullptr;
    rc = get_alpha(ctx, iters, &alpha);
    if (rc) return rc;
    const long long N = (long long)ny * nx;
    // byte masks followed (16-byte aligned) by per-mask bits of the kx columns
    // and of the ky rows that hold any sample
    const int cw = (nx + 31) / 32, rw = (ny + 31) / 32;
    const size_t mbytes = (size_t)nmask * N, cb_off = (mbytes + 15) & ~size_t(15);
    const size_t rb_off = cb_off + sizeof(uint32_t) * (size_t)nmask * cw;
    const size_t up_bytes = rb_off + sizeof(uint32_t) * (size_t)nmask * rw;
    if (ctx->h_mask_up.size() < up_bytes) ctx->h_mask_up.resize(up_bytes);   // kept across calls
    uint8_t* up = ctx->h_mask_up.data();
    std::memcpy(up, h_mask, mbytes);
    std::memset(up + mbytes, 0, up_bytes - mbytes);
    uint32_t* colbits = reinterpret_cast<uint32_t*>(up + cb_off);
    uint32_t* rowbits = reinterpret_cast<uint32_t*>(up + rb_off);
    // per mask: the rows with any sample, the OR of those rows (the columns
    // with any sample), and whether every sampled row holds exactly those
    // columns (separable).  Whole-row loops the compiler vectorises; the
    // byte-exact test runs only for a row whose bytes differ from the OR.
    bool separable = true;
    std::vector<uint8_t> any_row((size_t)nx);
    for (int k = 0; k < nmask; ++k) {
        const uint8_t* mk = h_mask + (size_t)k * N;
        std::fill(any_row.begin(), any_row.end(), uint8_t(0));
        for (int r = 0; r < ny; ++r) {
            const uint8_t* row = mk + (size_t)r * nx;
            uint8_t acc = 0;
            for (int x = 0; x < nx; ++x) acc |= row[x];
            if (!acc) continue;
            rowbits[(size_t)k * rw + (r >> 5)] |= 1u << (r & 31);
            for (int x = 0; x < nx; ++x) any_row[x] |= row[x];
        }
        for (int x = 0; x < nx; ++x)
            if (any_row[x]) colbits[(size_t)k * cw + (x >> 5)] |= 1u << (x & 31);
        for (int r = 0; r < ny && separable; ++r) {
            if (!((rowbits[(size_t)k * rw + (r >> 5)] >> (r & 31)) & 1u)) continue;
            const uint8_t* row = mk + (size_t)r * nx;
            if (std::memcmp(row, any_row.data(), (size_t)nx) == 0) continue;
            for (int x = 0; x < nx; ++x)
                if ((row[x] != 0) != (any_row[x] != 0)) {
                    separable = false;
                    break;
                }
        }
    }
    oks::Staging::Slot* slot = nullptr;
    rc = stage_upload(ctx, up, up_bytes, &slot);
    if (rc) return rc;
    const TuneParams tp = tune_params(ctx, 1, ny, nx);
    long long chunk = tp.fista2d_chunk > 0 ? tp.fista2d_chunk
                                             : std::max<long long>(1, (96ll << 20) / (4 * N * 8));
    if (chunk > nprob) chunk = nprob;
    // independent chunks run concurrently on `ns` forked streams, each with
    // its own state, so that one chunk's launch tails overlap the other's
    const long long nchunks = (nprob + chunk - 1) / chunk;
    const int ns = (int)std::max<long long>(1, std::min<long long>(tp.fista2d_streams, nchunks));
    // row pass on the tensor cores (row_engine 1): F_x^H restricted to the kx
    // columns any mask samples, prox, F_x back onto those columns
    const bool use_tc = ctx->row_engine == 1;
    std::vector<int> tcols;
    const okscuda_ctx::TcMat *m_inv = nullptr, *m_fwd = nullptr;
    size_t per_stream = 3 * (size_t)chunk * N;   // float2 elements: Z, S, X
    size_t tc_split = 0;                           // bytes of bf16 split operands per stream
    if (use_tc) {
        if (nx > 2048 || !oks::dft_tc_available() || (long long)chunk * ny > 65535ll * 128) {
            stage_release(ctx, slot);
            return set_err(ctx, OKS_ENOTSUP, "row_engine 1: tensor-core row DFT unavailable for nx = %d", nx);
        }
        for (int x = 0; x < nx; ++x) {
            bool any = false;
            for (int k = 0; k < nmask && !any; ++k) any = (colbits[(size_t)k * cw + (x >> 5)] >> (x & 31)) & 1u;
            if (any) tcols.push_back(x);
        }
        if (tcols.empty()) tcols.push_back(0);   // nothing sampled: one (zero) column keeps the GEMMs non-empty
        if ((rc = tc_matrix(ctx, nx, +1, 0, tcols, {}, &m_inv)) || (rc = tc_matrix(ctx, nx, -1, 0, {}, tcols, &m_fwd)) ||
            (rc = tc_err_flag(ctx))) {
            stage_release(ctx, slot);
            return rc;
        }
        per_stream += (size_t)chunk * N;   // W = F_x^H S
        tc_split = std::max(oks::dft_tc_scratch_bytes(chunk * ny, (int)tcols.size()),
                            oks::dft_tc_scratch_bytes(chunk * ny, nx));
        tc_split = (tc_split + 255) & ~size_t(255);
    }
    const size_t stream_bytes = ((sizeof(float2) * per_stream + 255) & ~size_t(255)) + tc_split;
    const int hs = ((ny / 2) + (nx / 2)) & 1;
    // register-resident passes where a compile-time plan exists (col_engine 1
    // forces the generic shared-memory passes)
    const bool col_reg = tp.col_engine != 1 && oks::fista2d_reg_supported(ny);
    const bool row_reg = tp.col_engine != 1 && oks::fista2d_reg_supported(nx);
    cudaError_t e = cudaSuccess;
    if (row_reg && (tp.prefetch2d & 4) && (rc = tc_err_flag(ctx))) {   // the bulk-copy row pass's error word
        stage_release(ctx, slot);
        return rc;
    }
    if ((col_reg || row_reg) && (e = oks::reg_tables_init(&ctx->reg_tables)) != cudaSuccess) {
        stage_release(ctx, slot);
        return cuda_err(ctx, e, "register tables");
    }
    if (ns > 1 && (rc = ensure_aux_streams(ctx, ns))) {
        stage_release(ctx, slot);
        return rc;
    }

    // The whole launch sequence of one call: chunks round-robin over `ns`
    // forked streams, every iteration's column and row pass, the demodulated
    // copy out.  Inputs, outputs, masks and scratch are parameters so that the
    // same sequence can be captured once into a CUDA graph over buffers the
    // graph owns (below).
    auto enqueue = [&](const float2* ysrc, float2* outdst, const uint8_t* mdev, void* scratch) -> cudaError_t {
        cudaError_t err = cudaSuccess;
        if (ns > 1) {
            if ((err = cudaEventRecord(ctx->fork_ev, ctx->stream)) != cudaSuccess) return err;
            for (int k = 0; k < ns; ++k)
                if ((err = cudaStreamWaitEvent(ctx->aux[k].stream, ctx->fork_ev, 0)) != cudaSuccess) return err;
        }
        long long ci = 0;
        for (long long p0 = 0; p0 < nprob && err == cudaSuccess; p0 += chunk, ++ci) {
            const int k = (int)(ci % ns);
            cudaStream_t st = ns > 1 ? ctx->aux[k].stream : ctx->stream;
            uint8_t* sbase = static_cast<uint8_t*>(scratch) + (size_t)k * stream_bytes;
            float2* base = reinterpret_cast<float2*>(sbase);
            float2* W = base + 3 * chunk * N;                                      // tensor-core mode only
            void* split = sbase + ((sizeof(float2) * per_stream + 255) & ~size_t(255));
            oks::Fista2dArgs a{};
            a.nprob = std::min(chunk, nprob - p0);
            a.y = ysrc + p0 * N;
            a.y_stride = N;
            // problem p0 + i uses mask (p0 + i) % nmask (mask_offset = p0 % nmask)
            a.mask_mod = nmask;
            a.mask_stride = N;
            a.mask = mdev;
            a.colbits = reinterpret_cast<const uint32_t*>(mdev + cb_off);
            a.col_wstride = cw;
            a.rowbits = reinterpret_cast<const uint32_t*>(mdev + rb_off);
            a.row_wstride = rw;
            a.separable = separable && ctx->mask_bits != 0;
            a.X = base + 2 * chunk * N;
            a.Z = base;
            a.S = a.Z + chunk * N;
            a.st_stride = N;
            a.ny = ny; a.nx = nx;
            a.ysc = std::sqrt((float)ny * (float)nx) * (hs ? -1.f : 1.f);
            a.minv = 1.0f / ((float)ny * (float)nx);
            a.lambda = lambda;
            a.alpha = alpha;
            a.mask_offset = p0 % nmask;
            a.persist = tp.persist2d;
            a.occ = tp.occ2d;
            a.prefetch = tp.prefetch2d;
            a.err = ctx->tc_err;
            // 0: by length -- the pruned two-stage form (14) at ny = 368 (it
            // takes the iteration passes of separable masks; the rest stay on
            // the column-pair pass), the column-pair pass elsewhere
            a.col_lanes = ctx->col2d_lanes > 0 ? ctx->col2d_lanes : (ctx->col2d_lanes == 0 && ny == 368 ? 14 : 0);
            a.row_ctas = ctx->row2d_ctas;
            a.pdl = ctx->pdl2d;
            a.col_ctas = ctx->col2d_ctas;
            auto col = [&](int mode) {
                if (col_reg) {
                    ProfScope ps(ctx, "k2d_col_reg", st);
                    return oks::launch_fista2d_col_reg(a, ctx->reg_tables, mode, st);
                }
                ProfScope ps(ctx, "k2d_col", st);
                return oks::launch_fista2d_col(a, *py, mode, st);
            };
            auto row = [&](int mode, int it) {
                if (use_tc) {
                    const bool contiguous = tcols.back() - tcols.front() + 1 == (int)tcols.size();
                    oks::DftTcArgs t{};
                    t.M = a.nprob * ny;
                    t.scale = 1.0f;
                    t.scratch = split;
                    t.err = ctx->tc_err;
                    // h = F_x^H S over the sampled columns
                    t.in = a.S; t.ld_in = nx; t.nin = (int)tcols.size();
                    t.in_cols = contiguous ? nullptr : m_inv->in_cols;
                    t.in_col0 = contiguous ? tcols.front() : 0;
                    t.out = W; t.ld_out = nx; t.nout = nx;
                    t.b_hi = m_inv->hi; t.b_lo = m_inv->lo;
                    cudaError_t e1;
                    {
                        ProfScope ps(ctx, "k_dft_tc", st);
                        e1 = oks::launch_dft_tc(t, st);
                    }
                    if (e1 != cudaSuccess) return e1;
                    {
                        ProfScope ps(ctx, "k2d_prox", st);
                        e1 = oks::launch_fista2d_prox(a, W, mode, it, st);
                    }
                    if (e1 != cudaSuccess) return e1;
                    // S = F_x z~' on the sampled columns, zero where the row's mask is clear
                    oks::DftTcArgs f = t;
                    f.in = a.Z; f.nin = nx; f.in_cols = nullptr; f.in_col0 = 0;
                    f.out = a.S; f.nout = (int)tcols.size();
                    f.out_cols = contiguous ? nullptr : m_fwd->out_cols;
                    f.out_col0 = contiguous ? tcols.front() : 0;
                    f.colbits = a.colbits; f.col_wstride = cw; f.rows_per_prob = ny;
                    f.mask_offset = a.mask_offset; f.mask_mod = nmask;
                    f.b_hi = m_fwd->hi; f.b_lo = m_fwd->lo;
                    ProfScope ps(ctx, "k_dft_tc", st);
                    return oks::launch_dft_tc(f, st);
                }
                if (row_reg) {
                    ProfScope ps(ctx, "k2d_row_reg", st);
                    return oks::launch_fista2d_row_reg(a, ctx->reg_tables, mode, it, st);
                }
                ProfScope ps(ctx, "k2d_row", st);
                return oks::launch_fista2d_row(a, *px, mode, it, st);
            };
            // the tensor-core row pass reads every sampled column of S, also
            // those of column pairs the column pass skips for this problem's mask
            if (use_tc) err = cudaMemsetAsync(a.S, 0, sizeof(float2) * a.nprob * N, st);
            if (err == cudaSuccess) err = col(0);
            if (err == cudaSuccess) err = row(0, 0);
            for (int it = 0; it < iters && err == cudaSuccess; ++it) {
                err = col(1);
                if (err == cudaSuccess) err = row(1, it);
            }
            if (err == cudaSuccess) {
                ProfScope ps(ctx, "k2d_demod", st);
                err = oks::launch_fista2d_demod(a.X, outdst + p0 * N, a.nprob, ny, nx, N, N, st);
            }
        }
        // join (also after a launch error)
        for (int k = 0; k < ns && ns > 1; ++k) {
            cudaEventRecord(ctx->aux[k].done, ctx->aux[k].stream);
            cudaStreamWaitEvent(ctx->stream, ctx->aux[k].done, 0);
        }
        return err;
    };

    // CUDA-graph form (graph2d, SIMT row engine): the second call with the
    // same shape, iterations, lambda and choices captures the launch sequence
    // over buffers owned by the cache entry; every later call copies its
    // k-space and masks in, replays the graph (one launch for all chunks and
    // iterations) and copies the coil images out.  The first call runs the
    // launches directly, which also creates every table the capture needs.
    const size_t data_bytes = sizeof(float2) * (size_t)nprob * N;
    if (ctx->graph2d && !use_tc) {
        char kb[320];
        std::snprintf(kb, sizeof kb, "%d/%d/%lld/%d/%d/%08x/%lld/%d/%d/%d/%d/%d/%d/%d/%d/%zu/%d/%d/%d/%d/%d", ny, nx, nprob, nmask,
                      iters, [&] { uint32_t u; std::memcpy(&u, &lambda, 4); return u; }(), chunk, ns, (int)col_reg,
                      (int)row_reg, tp.persist2d, tp.occ2d, tp.prefetch2d, (int)separable, ctx->mask_bits, up_bytes,
                      ctx->device, ctx->col2d_lanes, ctx->row2d_ctas, ctx->col2d_ctas, ctx->pdl2d);
        const std::string key(kb);
        auto it = ctx->g2d.find(key);
        if (it == ctx->g2d.end()) {
            ctx->g2d.emplace(key, okscuda_ctx::Graph2d{});   // seen once: run directly this time
        } else if (!it->second.failed) {
            okscuda_ctx::Graph2d& g = it->second;
            g.last_use = ++ctx->g2d_clock;
            if (!g.exec) {
                // evict the least recently used entry beyond the cache size
                if (ctx->g2d.size() > 4) {
                    auto victim = ctx->g2d.end();
                    for (auto v = ctx->g2d.begin(); v != ctx->g2d.end(); ++v)
                        if (v != it && (victim == ctx->g2d.end() || v->second.last_use < victim->second.last_use))
                            victim = v;
                    if (victim != ctx->g2d.end()) {
                        cudaDeviceSynchronize();
                        free_graph2d(victim->second);
                        ctx->g2d.erase(victim);
                    }
                }
                cudaError_t ge = cudaMalloc(&g.y, data_bytes);
                if (ge == cudaSuccess) ge = cudaMalloc(&g.out, data_bytes);
                if (ge == cudaSuccess) ge = cudaMalloc(&g.masks, up_bytes);
                if (ge == cudaSuccess) ge = cudaMalloc(&g.scratch, stream_bytes * ns);
                if (ge == cudaSuccess) ge = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
                if (ge == cudaSuccess) {
                    const bool prof = ctx->prof_on;
                    ctx->prof_on = false;
                    cudaGraph_t graph = nullptr;
                    ge = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
                    if (ge == cudaSuccess) {
                        cudaError_t le = enqueue(static_cast<const float2*>(g.y), static_cast<float2*>(g.out),
                                                 static_cast<const uint8_t*>(g.masks), g.scratch);
                        ge = cudaStreamEndCapture(ctx->stream, &graph);
                        if (le != cudaSuccess) ge = le;
                    }
                    if (ge == cudaSuccess) {
                        // count the kernel nodes, so profiling reports the kernels a replay runs
                        size_t nn = 0;
                        if (cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn > 0) {
                            std::vector<cudaGraphNode_t> nodes(nn);
                            if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
                                for (size_t q = 0; q < nn; ++q) {
                                    cudaGraphNodeType ty;
                                    if (cudaGraphNodeGetType(nodes[q], &ty) == cudaSuccess &&
                                        ty == cudaGraphNodeTypeKernel)
                                        ++g.kernels;
                                }
                        }
                        ge = cudaGraphInstantiate(&g.exec, graph, 0);
                    }
                    if (graph) cudaGraphDestroy(graph);
                    ctx->prof_on = prof;
                }
                if (ge != cudaSuccess) {
                    (void)cudaGetLastError();
                    free_graph2d(g);
                    g.failed = true;   // this shape keeps the direct launches
                }
            }
            if (g.exec) {
                cudaError_t ge = cudaStreamWaitEvent(ctx->stream, g.done, 0);   // the previous replay is done
                if (ge == cudaSuccess)
                    ge = cudaMemcpyAsync(g.masks, slot->dev, up_bytes, cudaMemcpyDeviceToDevice, ctx->stream);
                if (ge == cudaSuccess)
                    ge = cudaMemcpyAsync(g.y, d_kspace, data_bytes, cudaMemcpyDeviceToDevice, ctx->stream);
                if (ge == cudaSuccess) {
                    ProfScope ps(ctx, "k2d_graph", nullptr, g.kernels > 0 ? g.kernels : 1);
                    ge = cudaGraphLaunch(g.exec, ctx->stream);
                }
                if (ge == cudaSuccess)
                    ge = cudaMemcpyAsync(d_out, g.out, data_bytes, cudaMemcpyDeviceToDevice, ctx->stream);
                if (ge == cudaSuccess) ge = cudaEventRecord(g.done, ctx->stream);
                stage_release(ctx, slot);
                if (ge != cudaSuccess) return cuda_err(ctx, ge, "fista2d graph replay");
                return OKS_OK;
            }
        }
    }

    void* scratch = nullptr;
    e = cudaMallocAsync(&scratch, stream_bytes * ns, ctx->stream);
    if (e != cudaSuccess) { stage_release(ctx, slot); return cuda_err(ctx, e, "cudaMallocAsync(fista2d)"); }
    e = enqueue(reinterpret_cast<const float2*>(d_kspace), reinterpret_cast<float2*>(d_out),
                static_cast<const uint8_t*>(slot->dev), scratch);
    cudaFreeAsync(scratch, ctx->stream);
    stage_release(ctx, slot);
    if (e != cudaSuccess) return cuda_err(ctx, e, "fista2d launch");
    return OKS_OK;
}

// FISTA on `nprob` problems [nprob][ny][nx]; problem b uses mask b % nmask.
int oks_fista_core(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nmask,
                      long long nprob, int ny, int nx, int iters, float lambda, okscuda_c64* d_out) {
    if (!h_mask || nmask <= 0 || nprob < 0 || ny <= 0 || nx <= 0 || iters < 0)
        return set_err(ctx, OKS_EINVAL, "fista_cs: bad arguments");
    if (ny % 2 || nx % 2)
        return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", ny, nx);
    if (nprob == 0) return OKS_OK;
    if (!d_kspace || !d_out) return set_err(ctx, OKS_EINVAL, "fista_cs: null data pointer");
    std::vector<uint32_t> words;
    int wstride = 0;
    if (!pack_row_masks(h_mask, nmask, ny, nx, &words, &wstride))
        return fista2d_core(ctx, d_kspace, h_mask, nmask, nprob, ny, nx, iters, lambda, d_out);
    const DevPlan *px, *py;
    int rc = get_plan(ctx, nx, &px);
    if (rc) return rc;
    rc = get_plan(ctx, ny, &py);
    if (rc) return rc;
    const float* alpha = nullptr;
    rc = get_alpha(ctx, iters, &alpha);
    if (rc) return rc;
    oks::Staging::Slot* slot = nullptr;
    rc = stage_upload(ctx, words.data(), words.size() * sizeof(uint32_t), &slot);
    if (rc) return rc;
    oks::RowMasks rm{static_cast<const uint32_t*>(slot->dev), wstride, nmask};

    // y' = sqrt(ny) (-1)^{ny/2} (-1)^r * centred unitary row-IDFT of y
    float2* out = reinterpret_cast<float2*>(d_out);
    oks::RowXformArgs ra{};
    ra.reg = ctx->xform_reg;
    ra.in = reinterpret_cast<const float2*>(d_kspace);
    ra.out = out;
    ra.nrows = nprob * ny;
    ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = +1; ra.centred = 1;
    ra.scale = std::sqrt((float)ny) / std::sqrt((float)nx) * (((ny / 2) & 1) ? -1.0f : 1.0f);
    ra.rows_per_prob = ny; ra.rowsign = 1;
    ra.use_keep = 1; ra.keep = rm;
    cudaError_t e;
    {
        ProfScope ps(ctx, "k_row_xform");
        e = oks::launch_row_xform(ra, *px, ctx->stream);
    }
    if (e == cudaSuccess) {
        oks::FistaColArgs fa{};
        fa.ytil = out; fa.prob_stride = (long long)ny * nx;
        fa.minv = 1.0f / (float)ny;
        fa.mask = rm;
        fa.xout = out; fa.out_stride = (long long)ny * nx;
        fa.ny = ny; fa.nx = nx; fa.iters = iters; fa.lambda = lambda; fa.alpha = alpha;
        fa.nprob = nprob;
        const TuneParams tp = tune_params(ctx, 0, ny, nx);
        fa.variant = tp.col_variant;
        const bool use_reg = tp.col_engine != 1 && oks::fista_col_reg_supported(ny);
        if (use_reg) e = oks::reg_tables_init(&ctx->reg_tables);
        if (e == cudaSuccess && use_reg) {
            ProfScope ps(ctx, "k_fista_col_reg");
            e = oks::launch_fista_col_reg(fa, ctx->reg_tables, ctx->stream);
        } else if (e == cudaSuccess) {
            ProfScope ps(ctx, "k_fista_col");
            e = oks::launch_fista_col(fa, *py, ctx->stream);
        }
    }
    stage_release(ctx, slot);
    if (e != cudaSuccess) return cuda_err(ctx, e, "fista_cs launch");
    return OKS_OK;
}

int okscuda_fista_cs(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int batch, int ny,
                     int nx, int iters, float lambda, okscuda_c64* d_out) {
    OKS_CHECK_CTX();
    return oks_fista_core(ctx, d_kspace, h_mask, 1, batch, ny, nx, iters, lambda, d_out);
}

int okscuda_cs_volume(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc, int nz,
                      int ny, int nx, int iters, float lambda, int ty, int tx, float* d_rss,
                      okscuda_c64* d_coils) {
    OKS_CHECK_CTX();
    if (!d_rss || nc < 0 || nz <= 0 || ty <= 0 || tx <= 0 || ty > ny || tx > nx)
        return set_err(ctx, OKS_EINVAL, "cs_volume: bad arguments");
    okscuda_c64* coils = d_coils;
    void* own = nullptr;
    const size_t bytes = sizeof(okscuda_c64) * (size_t)nc * nz * ny * nx;
    if (!coils && bytes) {
        OKS_CUDA(cudaMallocAsync(&own, bytes, ctx->stream));
        coils = static_cast<okscuda_c64*>(own);
    }
    int rc = oks_fista_core(ctx, d_kspace, h_mask, nz, (long long)nc * nz, ny, nx, iters, lambda, coils);
    if (rc == OKS_OK) {
        oks::RssArgs a{};
        a.coils = reinterpret_cast<const float2*>(coils);
        a.coil_stride = (long long)nz * ny * nx;
        a.nc = nc; a.ny = ny; a.nx = nx;
        a.nslice = nz; a.slice_stride = (long long)ny * nx;
        a.ty = ty; a.tx = tx; a.y0 = (ny - ty) / 2; a.x0 = (nx - tx) / 2;
        a.out = d_rss;
        ProfScope ps(ctx, "k_rss");
        cudaError_t e = oks::launch_rss(a, ctx->stream);
        if (e != cudaSuccess) rc = cuda_err(ctx, e, "rss");
    }
    if (own) cudaFreeAsync(own, ctx->stream);
    return rc;
}

int okscuda_cs_slice(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc, int ny,
                     int nx, int iters, float lambda, float* d_rss, okscuda_c64* d_coils) {
    return okscuda_cs_volume(ctx, d_kspace, h_mask, nc, 1, ny, nx, iters, lambda, ny, nx, d_rss, d_coils);
}

// ---------------------------------------------------------------- profiling
int okscuda_profile_enable(okscuda_ctx* ctx, int on) {
    OKS_CHECK_CTX();
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto& r : ctx->prof) { ctx->ev_pool.push_back(r.a); ctx->ev_pool.push_back(r.b); }
    ctx->prof.clear();
    ctx->prof_on = on != 0;
    return OKS_OK;
}

int okscuda_profile_read(okscuda_ctx* ctx, char* names, int name_len, double* total_ms, long long* launches,
                         int nslots, int* nfound) {
    OKS_CHECK_CTX();
    if (!nfound) return set_err(ctx, OKS_EINVAL, "profile_read: null count");
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<std::string> keys;
    std::vector<double> ms;
    std::vector<long long> cnt;
    for (auto& r : ctx->prof) {
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        size_t k = 0;
        for (; k < keys.size(); ++k)
            if (keys[k] == r.name) break;
        if (k == keys.size()) { keys.push_back(r.name); ms.push_back(0.0); cnt.push_back(0); }
        ms[k] += t;
        cnt[k] += r.kernels;
    }
    *nfound = (int)keys.size();
    for (int k = 0; k < (int)keys.size() && k < nslots; ++k) {
        if (names && name_len > 0) std::snprintf(names + (size_t)k * name_len, name_len, "%s", keys[k].c_str());
        if (total_ms) total_ms[k] = ms[k];
        if (launches) launches[k] = cnt[k];
    }
    return OKS_OK;
}

}  // extern "C"
