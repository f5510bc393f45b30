// Row transforms along the readout direction through the C-ABI: the SIMT
// mixed-radix FFT (k_row_xform) and its tensor-core counterpart, the DFT as
// one split-precision 3xBF16 GEMM on tcgen05 (k_dft_tc.cu).  Same meaning as
// the reference's per-row rustfft call inside centred_fft2 (cs.rs:141-178),
// unnormalised, with the fftshift/ifftshift pair when `centred` is set.
#include "ctx.h"

namespace {

int tc_matrix(okscuda_ctx* ctx, int n, int sign, int centred, const void** hi, const void** lo) {
    const long long key = ((long long)n << 2) | ((sign > 0) << 1) | (centred != 0);
    auto it = ctx->tc_mats.find(key);
    if (it == ctx->tc_mats.end()) {
        std::vector<uint16_t> h, l;
        oks::tc::dft_matrix_split(n, sign, centred, &h, &l);
        okscuda_ctx::TcMat m;
        const size_t bytes = h.size() * sizeof(uint16_t);
        OKS_CUDA(cudaMalloc(&m.hi, bytes));
        cudaError_t e = cudaMalloc(&m.lo, bytes);
        if (e != cudaSuccess) { cudaFree(m.hi); return cuda_err(ctx, e, "cudaMalloc(dft matrix)"); }
        // pageable source: the copies complete before cudaMemcpy returns
        if ((e = cudaMemcpy(m.hi, h.data(), bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(m.lo, l.data(), bytes, cudaMemcpyHostToDevice)) != cudaSuccess) {
            cudaFree(m.hi);
            cudaFree(m.lo);
            return cuda_err(ctx, e, "dft matrix upload");
        }
        it = ctx->tc_mats.emplace(key, m).first;
    }
    *hi = it->second.hi;
    *lo = it->second.lo;
    return OKS_OK;
}

int tc_err_flag(okscuda_ctx* ctx) {
    if (!ctx->tc_err) {
        OKS_CUDA(cudaMalloc(&ctx->tc_err, sizeof(int)));
        OKS_CUDA(cudaMemset(ctx->tc_err, 0, sizeof(int)));
    }
    return OKS_OK;
}

}  // namespace

extern "C" int okscuda_dft_rows(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, long long nrows,
                                int n, int inverse, int centred, int engine) {
    OKS_CHECK_CTX();
    if (!d_in || !d_out || nrows < 0 || n <= 0 || (engine != 0 && engine != 1))
        return set_err(ctx, OKS_EINVAL, "dft_rows: bad arguments");
    if (nrows == 0) return OKS_OK;
    const int sign = inverse ? +1 : -1;
    if (engine == 0) {
        const DevPlan* px;
        int rc = get_plan(ctx, n, &px);
        if (rc) return rc;
        oks::RowXformArgs ra{};
        ra.in = reinterpret_cast<const float2*>(d_in);
        ra.out = reinterpret_cast<float2*>(d_out);
        ra.nrows = nrows;
        ra.ld_in = n; ra.ld_out = n;
        ra.sign = sign; ra.centred = centred != 0; ra.scale = 1.0f;
        ra.rows_per_prob = 1;
        ProfScope ps(ctx, "k_row_xform");
        OKS_CUDA(oks::launch_row_xform(ra, *px, ctx->stream));
        return OKS_OK;
    }
    if (n > 2048) return set_err(ctx, OKS_ENOTSUP, "dft_rows: tensor-core engine supports n <= 2048 (n = %d)", n);
    if (nrows > 65535ll * 128)
        return set_err(ctx, OKS_ENOTSUP, "dft_rows: tensor-core engine takes at most %lld rows per call",
                       65535ll * 128);
    if (!oks::dft_tc_available())
        return set_err(ctx, OKS_ENOTSUP, "dft_rows: cuTensorMapEncodeTiled is not available from the driver");
    const void *bhi, *blo;
    int rc = tc_matrix(ctx, n, sign, centred, &bhi, &blo);
    if (rc) return rc;
    if ((rc = tc_err_flag(ctx))) return rc;
    void* scratch = nullptr;
    OKS_CUDA(cudaMallocAsync(&scratch, oks::dft_tc_scratch_bytes(nrows, n), ctx->stream));
    cudaError_t e;
    {
        ProfScope ps(ctx, "k_dft_tc");
        e = oks::launch_dft_tc(reinterpret_cast<const float2*>(d_in), n, reinterpret_cast<float2*>(d_out), n, nrows,
                               n, bhi, blo, scratch, 1.0f, ctx->tc_err, ctx->stream);
    }
    cudaFreeAsync(scratch, ctx->stream);
    if (e != cudaSuccess) return cuda_err(ctx, e, "dft_rows (tensor cores)");
    return OKS_OK;
}

extern "C" int okscuda_tc_status(okscuda_ctx* ctx, int* status) {
    OKS_CHECK_CTX();
    if (!status) return set_err(ctx, OKS_EINVAL, "tc_status: null pointer");
    *status = 0;
    if (!ctx->tc_err) return OKS_OK;
    OKS_CUDA(cudaMemcpyAsync(status, ctx->tc_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    OKS_CUDA(cudaMemsetAsync(ctx->tc_err, 0, sizeof(int), ctx->stream));
    return OKS_OK;
}
