// Row transforms along the readout direction through the C-ABI: the SIMT
// mixed-radix FFT (k_row_xform) and its tensor-core counterpart, the DFT as
// one split-precision 3xBF16 GEMM on tcgen05 (k_dft_tc.cu).  Same meaning as
// the reference's per-row rustfft call inside centred_fft2 (cs.rs:141-178),
// unnormalised, with the fftshift/ifftshift pair when `centred` is set.
#include "ctx.h"

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
        ra.reg = ctx->xform_reg;
        ra.variant = ctx->xform_row_variant;
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
    const okscuda_ctx::TcMat* mat;
    int rc = tc_matrix(ctx, n, sign, centred != 0, {}, {}, &mat);
    if (rc) return rc;
    if ((rc = tc_err_flag(ctx))) return rc;
    void* scratch = nullptr;
    OKS_CUDA(cudaMallocAsync(&scratch, oks::dft_tc_scratch_bytes(nrows, n), ctx->stream));
    oks::DftTcArgs a{};
    a.in = reinterpret_cast<const float2*>(d_in);
    a.ld_in = n; a.nin = n;
    a.out = reinterpret_cast<float2*>(d_out);
    a.ld_out = n; a.nout = n;
    a.M = nrows;
    a.scale = 1.0f;
    a.b_hi = mat->hi; a.b_lo = mat->lo;
    a.scratch = scratch;
    a.err = ctx->tc_err;
    if (ctx->tc_gate_cycles > 0) {   // bounded-wait test: a gate that never opens
        a.gate = ctx->tc_err + 1;
        a.gate_cycles = ctx->tc_gate_cycles;
    }
    cudaError_t e;
    {
        ProfScope ps(ctx, "k_dft_tc");
        e = oks::launch_dft_tc(a, ctx->stream);
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
