// okscuda_sense_cs: the SENSE extension mode for one slice -- Walsh maps from
// the ACS block, an FP64 power-iteration estimate of L = ||A||^2, then FISTA
// on one coil-combined image with step 1/L (SENSE-map expand/combine inside
// every iteration).  The reference's cs strategy has no counterpart (it is
// per-coil; cs.rs:23-26); the map estimate follows sensitivity.rs:37-142
// and SenseRss (strategy.rs:656-671), the ACS block grappa.rs:50-87.
#include "ctx.h"

namespace {

// grappa.rs:50-87: longest run of consecutive sampled rows (first longest)
bool acs_block(const std::vector<uint8_t>& rows, int* a0, int* a1) {
    std::vector<int> s;
    for (int i = 0; i < (int)rows.size(); ++i)
        if (rows[i]) s.push_back(i);
    if (s.size() < 4) return false;
    int best_start = 0, best_len = 0, cur_start = s[0], cur_len = 1;
    for (size_t k = 1; k < s.size(); ++k) {
        if (s[k] == s[k - 1] + 1) ++cur_len;
        else {
            if (cur_len > best_len) { best_len = cur_len; best_start = cur_start; }
            cur_start = s[k];
            cur_len = 1;
        }
    }
    if (cur_len > best_len) { best_len = cur_len; best_start = cur_start; }
    *a0 = best_start;
    *a1 = best_start + best_len;
    return true;
}

}  // namespace

extern "C" int okscuda_sense_cs(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc, int ny,
                                int nx, int iters, float lambda, int walsh_window, int walsh_iters, int power_iters,
                                float* d_mag, okscuda_c64* d_maps, okscuda_c64* d_x, double* h_lipschitz) {
    OKS_CHECK_CTX();
    if (!d_kspace || !h_mask || !d_mag || nc <= 0 || ny <= 0 || nx <= 0 || iters < 0 || walsh_window < 0 ||
        walsh_iters < 0 || power_iters < 1)
        return set_err(ctx, OKS_EINVAL, "sense_cs: bad arguments");
    if (ny % 2 || nx % 2)
        return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", ny, nx);
    if (nc > 32) return set_err(ctx, OKS_ENOTSUP, "sense_cs: nc=%d above 32", nc);
    if (!oks::sense_reg_supported(ny)) return set_err(ctx, OKS_ENOTSUP, "sense_cs: no plan for ny=%d", ny);
    // ky-only mask
    std::vector<uint8_t> rows(ny, 0);
    for (int r = 0; r < ny; ++r) {
        const uint8_t* m = h_mask + (size_t)r * nx;
        for (int x = 1; x < nx; ++x)
            if ((m[x] != 0) != (m[0] != 0)) return set_err(ctx, OKS_ENOTSUP, "sense_cs: mask varies along kx");
        rows[r] = m[0] != 0;
    }
    int a0 = 0, a1 = 0;
    if (!acs_block(rows, &a0, &a1)) return set_err(ctx, OKS_EINVAL, "sense_cs: fewer than 4 sampled rows (no ACS)");
    const DevPlan* px;
    int rc = get_plan(ctx, nx, &px);
    if (rc) return rc;
    const float* alpha = nullptr;
    if ((rc = get_alpha(ctx, iters, &alpha))) return rc;
    const long long N = (long long)ny * nx;
    const int wstride = (ny + 31) / 32;
    // host tables: row bits, FP64 twiddles e^{-2 pi i k / ny}
    const size_t tw_off = ((size_t)wstride * 4 + 15) & ~size_t(15);
    std::vector<uint8_t> up(tw_off + sizeof(double2) * ny, 0);
    uint32_t* words = reinterpret_cast<uint32_t*>(up.data());
    for (int r = 0; r < ny; ++r)
        if (rows[r]) words[r >> 5] |= 1u << (r & 31);
    double2* wt = reinterpret_cast<double2*>(up.data() + tw_off);
    for (int k = 0; k < ny; ++k) {
        const double ang = -6.283185307179586476925286766559 * k / ny;
        wt[k] = make_double2(std::cos(ang), std::sin(ang));
    }
    oks::Staging::Slot* slot = nullptr;
    if ((rc = stage_upload(ctx, up.data(), up.size(), &slot))) return rc;
    const uint32_t* d_words = static_cast<const uint32_t*>(slot->dev);
    const double2* d_wt = reinterpret_cast<const double2*>(static_cast<const uint8_t*>(slot->dev) + tw_off);

    // scratch: low-res images / y' (nc N c64), maps (if not given), FP64 v, acc, norms
    const size_t cN = (size_t)nc * N;
    void* scratch = nullptr;
    const size_t bytes = sizeof(float2) * cN * (d_maps ? 1 : 2) + sizeof(double2) * 2 * N + sizeof(double) * power_iters;
    cudaError_t e = cudaMallocAsync(&scratch, bytes, ctx->stream);
    if (e != cudaSuccess) { stage_release(ctx, slot); return cuda_err(ctx, e, "sense_cs scratch"); }
    float2* work = static_cast<float2*>(scratch);
    float2* maps = d_maps ? reinterpret_cast<float2*>(d_maps) : work + cN;
    double2* v = reinterpret_cast<double2*>(work + cN * (d_maps ? 1 : 2));
    double2* acc = v + N;
    double* norms = reinterpret_cast<double*>(acc + N);
    auto fail = [&](cudaError_t err, const char* where) {
        cudaFreeAsync(scratch, ctx->stream);
        stage_release(ctx, slot);
        return cuda_err(ctx, err, where);
    };
    // 1. low-resolution coil images: ACS rows only, centred IFFT2 (strategy.rs:658-669)
    if ((e = cudaMemsetAsync(work, 0, sizeof(float2) * cN, ctx->stream)) != cudaSuccess) return fail(e, "memset");
    e = cudaMemcpy2DAsync(work + (size_t)a0 * nx, sizeof(float2) * N, d_kspace + (size_t)a0 * nx, sizeof(float2) * N,
                          sizeof(float2) * (size_t)(a1 - a0) * nx, nc, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return fail(e, "ACS copy");
    if ((rc = okscuda_ifft2(ctx, reinterpret_cast<okscuda_c64*>(work), nc, ny, nx))) {
        cudaFreeAsync(scratch, ctx->stream);
        stage_release(ctx, slot);
        return rc;
    }
    // 2. Walsh maps, normalised to unit root-sum-of-squares
    {
        ProfScope ps(ctx, "k_walsh");
        if ((e = oks::launch_walsh(work, maps, nc, ny, nx, walsh_window, walsh_iters, 1, ctx->stream)) != cudaSuccess)
            return fail(e, "walsh");
    }
    // 3. L = ||A||^2 by FP64 power iteration on A^H A
    {
        ProfScope ps(ctx, "k_sense_normal_fp64");
        if ((e = cudaMemsetAsync(norms, 0, sizeof(double) * power_iters, ctx->stream)) != cudaSuccess)
            return fail(e, "memset");
        e = oks::launch_sense_power(maps, d_words, nc, ny, nx, power_iters, v, acc, d_wt, norms, ctx->stream);
        if (e != cudaSuccess) return fail(e, "power iteration");
    }
    double n2 = 0.0;
    if ((e = cudaMemcpyAsync(&n2, norms + power_iters - 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return fail(e, "norm read-back");
    double L = std::sqrt(n2);
    if (!(L > 0.0)) L = 1.0;
    if (h_lipschitz) *h_lipschitz = L;
    // 4. y'_c for every coil (row IDFT of the masked data, as the per-coil path)
    oks::RowXformArgs ra{};
    ra.reg = ctx->xform_reg;
    ra.in = reinterpret_cast<const float2*>(d_kspace);
    ra.out = work;
    ra.nrows = (long long)nc * ny;
    ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = +1; ra.centred = 1;
    ra.scale = std::sqrt((float)ny) / std::sqrt((float)nx) * (((ny / 2) & 1) ? -1.0f : 1.0f);
    ra.rows_per_prob = ny; ra.rowsign = 1;
    ra.use_keep = 1;
    ra.keep = oks::RowMasks{d_words, wstride, 1};
    {
        ProfScope ps(ctx, "k_row_xform");
        if ((e = oks::launch_row_xform(ra, *px, ctx->stream)) != cudaSuccess) return fail(e, "row pass");
    }
    // 5. SENSE FISTA
    oks::SenseArgs sa{};
    sa.ytil = work; sa.maps = maps;
    sa.nc = nc; sa.ny = ny; sa.nx = nx; sa.iters = iters;
    sa.minv = 1.0f / (float)ny;
    sa.lambda_l = (float)(lambda / L);
    sa.inv_l = (float)(1.0 / L);
    sa.mask = oks::RowMasks{d_words, wstride, 1};
    sa.alpha = alpha;
    sa.xout = reinterpret_cast<float2*>(d_x);
    sa.mag = d_mag;
    {
        ProfScope ps(ctx, "k_sense_col_reg");
        if ((e = oks::launch_sense_col_reg(sa, ctx->stream)) != cudaSuccess) return fail(e, "sense kernel");
    }
    cudaFreeAsync(scratch, ctx->stream);
    stage_release(ctx, slot);
    return OKS_OK;
}
