// Host side of the drop-in CsRss strategy (strategy.rs:736-892) and the
// C-ABI entry points of the feeding stages.  Geometry and bookkeeping (which
// acquisition lands where, the filled mask, output shape) are decided on the
// host from the acquisition headers, exactly as the reference's reader does;
// every pass over sample data runs in the sm_100a kernels.
#include "ctx.h"
#include "feed.h"

namespace {

// acquisition.rs:69-95 flag bits
constexpr uint64_t ACQ_IS_NOISE_MEASUREMENT = 1ull << (19 - 1);
constexpr uint64_t ACQ_IS_REVERSE = 1ull << (22 - 1);
constexpr uint64_t ACQ_IS_NAVIGATION_DATA = 1ull << (23 - 1);
constexpr uint64_t ACQ_IS_PHASECORR_DATA = 1ull << (24 - 1);
constexpr uint64_t ACQ_IS_HPFEEDBACK_DATA = 1ull << (26 - 1);
constexpr uint64_t ACQ_IS_DUMMYSCAN_DATA = 1ull << (27 - 1);
constexpr uint64_t ACQ_IS_RTFEEDBACK_DATA = 1ull << (28 - 1);
constexpr uint64_t ACQ_IS_SURFACECOILCORRECTIONSCAN_DATA = 1ull << (29 - 1);
constexpr uint64_t NON_IMAGE_MASK = ACQ_IS_NOISE_MEASUREMENT | ACQ_IS_PHASECORR_DATA | ACQ_IS_NAVIGATION_DATA |
                                    ACQ_IS_RTFEEDBACK_DATA | ACQ_IS_HPFEEDBACK_DATA | ACQ_IS_DUMMYSCAN_DATA |
                                    ACQ_IS_SURFACECOILCORRECTIONSCAN_DATA;

inline bool is_image(const okscuda_acq_header& h) { return (h.flags & NON_IMAGE_MASK) == 0; }

// oversampling.rs:50-71
bool os_ratio_ok(int enc, int rec) {
    if (rec <= 0 || enc <= rec || enc % rec != 0) return false;
    return enc / rec <= 8;
}

inline size_t sat_sub(size_t a, size_t b) { return a > b ? a - b : 0; }

// Device buffer released at scope exit (stream-ordered).
struct DevBuf {
    okscuda_ctx* ctx;
    void* p = nullptr;
    explicit DevBuf(okscuda_ctx* c) : ctx(c) {}
    cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes ? bytes : 16, ctx->stream); }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, ctx->stream);
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace

// The noise fit's launches (FP64 covariance, Cholesky, inverse); the result
// word (0 ok, 1 / 2 not positive definite) is left in d_status on the device.
// Errors the host can decide (sizes) are returned here.
static int prewhiten_fit_launch(okscuda_ctx* ctx, const okscuda_c64* d_noise, int nc, long long ns,
                                long long total_samples, okscuda_c64* d_W, int* d_status) {
    if (!d_W || nc <= 0 || ns < 0) return set_err(ctx, OKS_EINVAL, "prewhiten_fit: bad arguments");
    if (nc > 128) return set_err(ctx, OKS_ENOTSUP, "prewhiten_fit: nc=%d above 128", nc);
    const long long total = total_samples > 0 ? total_samples : ns;
    if (total < nc)
        return set_err(ctx, OKS_ESKIP, "Noise calibration: only %lld samples for %d channels -- skipping", total, nc);
    if (ns > 0 && !d_noise) return set_err(ctx, OKS_EINVAL, "prewhiten_fit: null noise");
    const int max_parts = 148 * 4;
    const size_t npair = (size_t)nc * (nc + 1) / 2;
    DevBuf part(ctx);   // released stream-ordered, after the kernels that use it
    OKS_CUDA(part.alloc(sizeof(double2) * npair * max_parts));
    // prewhiten.rs:98: denominator (total - 1).max(1)
    const double denom = std::max((double)total - 1.0, 1.0);
    ProfScope ps(ctx, "k_noise_fit");
    OKS_CUDA(oks::launch_noise_fit(reinterpret_cast<const float2*>(d_noise), nc, ns, denom, part.as<double2>(),
                                   max_parts, reinterpret_cast<float2*>(d_W), nullptr, d_status, ctx->stream));
    return OKS_OK;
}

extern "C" {

// ------------------------------------------------------- feeding stages
int okscuda_prewhiten_fit(okscuda_ctx* ctx, const okscuda_c64* d_noise, int nc, long long ns,
                          long long total_samples, okscuda_c64* d_W) {
    OKS_CHECK_CTX();
    DevBuf st(ctx);
    OKS_CUDA(st.alloc(sizeof(int)));
    int rc = prewhiten_fit_launch(ctx, d_noise, nc, ns, total_samples, d_W, st.as<int>());
    if (rc) return rc;
    int status = -1;
    OKS_CUDA(cudaMemcpyAsync(&status, st.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (status == 1) return set_err(ctx, OKS_ENOTPD, "Cholesky: non-positive-definite noise covariance");
    if (status == 2) return set_err(ctx, OKS_ENOTPD, "triangular inverse: singular diagonal");
    if (status != 0) return set_err(ctx, OKS_ECUDA, "prewhiten_fit: no status");
    return OKS_OK;
}

int okscuda_prewhiten_apply(okscuda_ctx* ctx, const okscuda_c64* d_W, okscuda_c64* d_data, long long nacq, int nc,
                            int ns) {
    OKS_CHECK_CTX();
    if (!d_W || (!d_data && nacq > 0) || nacq < 0 || nc <= 0 || ns < 0)
        return set_err(ctx, OKS_EINVAL, "prewhiten_apply: bad arguments");
    if (nc > 64) return set_err(ctx, OKS_ENOTSUP, "prewhiten_apply: nc=%d above 64", nc);
    int rc;
    if (ctx->prewhiten_bulk && (rc = tc_err_flag(ctx))) return rc;
    ProfScope ps(ctx, oks::prewhiten_bulk_eligible(reinterpret_cast<float2*>(d_data), nc, ns, ctx->tc_err,
                                                   ctx->prewhiten_bulk)
                          ? "k_prewhiten_bulk"
                          : "k_prewhiten_apply");
    OKS_CUDA(oks::launch_prewhiten_apply(reinterpret_cast<float2*>(d_data), reinterpret_cast<const float2*>(d_W),
                                         nacq, nc, ns, ctx->stream, nullptr, ctx->tc_err, ctx->prewhiten_bulk));
    return OKS_OK;
}

int okscuda_os_remove(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, long long nlines, int enc,
                      int rec) {
    OKS_CHECK_CTX();
    if (nlines < 0 || (nlines > 0 && (!d_in || !d_out)))
        return set_err(ctx, OKS_EINVAL, "os_remove: bad arguments");
    if (!os_ratio_ok(enc, rec))
        return set_err(ctx, OKS_ESKIP, "oversampling removal: %d -> %d is not an integer ratio in 2..8", enc, rec);
    const DevPlan *pe, *pr;
    int rc = get_plan(ctx, enc, &pe);
    if (rc) return rc;
    rc = get_plan(ctx, rec, &pr);
    if (rc) return rc;
    ProfScope ps(ctx, "k_os_remove");
    OKS_CUDA(oks::launch_os_remove(reinterpret_cast<const float2*>(d_in), reinterpret_cast<float2*>(d_out), nlines,
                                   *pe, *pr, ctx->stream));
    return OKS_OK;
}

int okscuda_ifft1_kz(okscuda_ctx* ctx, okscuda_c64* d_data, int nc, int nz, int ny, int nx) {
    OKS_CHECK_CTX();
    if (!d_data || nc < 0 || nz <= 0 || ny <= 0 || nx <= 0) return set_err(ctx, OKS_EINVAL, "ifft1_kz: bad arguments");
    if (nz < 2 || nc == 0) return OKS_OK;   // fft.rs:55 n < 2 is a no-op
    const DevPlan* pz;
    int rc = get_plan(ctx, nz, &pz);
    if (rc) return rc;
    oks::ColXformArgs ca{};
    ca.reg = ctx->xform_reg; ca.tile = ctx->xform_tile; ca.lanes = ctx->xform_lanes; ca.lanes_pf = ctx->xform_lanes_pf;
    ca.data = reinterpret_cast<float2*>(d_data);
    ca.nprob = nc;
    ca.ny = nz;
    ca.nx = ny * nx;
    ca.prob_stride = (long long)nz * ny * nx;
    ca.sign = +1;
    ca.centred = 1;
    ca.scale = 1.0f / (float)nz;
    ProfScope ps(ctx, "k_col_xform");
    OKS_CUDA(oks::launch_col_xform(ca, *pz, ctx->stream));
    return OKS_OK;
}

int okscuda_ifft2(okscuda_ctx* ctx, okscuda_c64* d_data, long long batch, int ny, int nx) {
    OKS_CHECK_CTX();
    if (!d_data || batch < 0 || ny <= 0 || nx <= 0) return set_err(ctx, OKS_EINVAL, "ifft2: bad arguments");
    if (batch == 0) return OKS_OK;
    float2* d = reinterpret_cast<float2*>(d_data);
    // fft.rs:59-84 skips n < 2 axes (no shift either: ifftshift of n=1 is the identity)
    if (ny >= 2) {
        const DevPlan* py;
        int rc = get_plan(ctx, ny, &py);
        if (rc) return rc;
        oks::ColXformArgs ca{};
        ca.reg = ctx->xform_reg; ca.tile = ctx->xform_tile; ca.lanes = ctx->xform_lanes; ca.lanes_pf = ctx->xform_lanes_pf;
        ca.data = d; ca.nprob = batch; ca.ny = ny; ca.nx = nx; ca.prob_stride = (long long)ny * nx;
        ca.sign = +1; ca.centred = 1; ca.scale = 1.0f / (float)ny;
        ProfScope ps(ctx, "k_col_xform");
        OKS_CUDA(oks::launch_col_xform(ca, *py, ctx->stream));
    }
    if (nx >= 2) {
        const DevPlan* px;
        int rc = get_plan(ctx, nx, &px);
        if (rc) return rc;
        oks::RowXformArgs ra{};
        ra.reg = ctx->xform_reg;
        ra.in = d; ra.out = d; ra.nrows = batch * ny; ra.ld_in = nx; ra.ld_out = nx;
        ra.sign = +1; ra.centred = 1; ra.scale = 1.0f / (float)nx; ra.rows_per_prob = ny;
        ProfScope ps(ctx, "k_row_xform");
        OKS_CUDA(oks::launch_row_xform(ra, *px, ctx->stream));
    }
    return OKS_OK;
}

// ---------------------------------------------------------------- CsRss
void okscuda_csrss_default(okscuda_csrss_cfg* cfg) {
    if (!cfg) return;
    cfg->remove_oversampling = 1;
    cfg->prewhiten = 1;
    cfg->phase_correct = 1;
    cfg->iters = 60;
    cfg->lambda = 0.01f;
    cfg->fft_mode = 0;
    cfg->crop_to_recon_matrix = 1;
}

const char* okscuda_csrss_name(void) { return "cs"; }
size_t okscuda_acq_header_size(void) { return sizeof(okscuda_acq_header); }
size_t okscuda_acq_set_size(void) { return sizeof(okscuda_acq_set); }

int okscuda_csrss_reconstruct(okscuda_ctx* ctx, const okscuda_csrss_cfg* cfg, const okscuda_acq_set* A,
                              float* h_out, long long out_cap, int* out_dims) {
    OKS_CHECK_CTX();
    if (!cfg || !A || !out_dims || (A->n_acq > 0 && (!A->headers || !A->data)))
        return set_err(ctx, OKS_EINVAL, "csrss_reconstruct: bad arguments");
    if (cfg->iters < 0) return set_err(ctx, OKS_EINVAL, "csrss_reconstruct: iters < 0");
    const okscuda_acq_header* H = A->headers;
    const long long nacq = A->n_acq;
    for (long long a = 0; a < nacq; ++a) {
        const long long need = H[a].data_offset + (long long)H[a].active_channels * H[a].number_of_samples;
        if (H[a].data_offset < 0 || need > A->data_len)
            return set_err(ctx, OKS_EINVAL, "acquisition %lld reaches past the data buffer", a);
    }
    const auto copy_kind = A->data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;

    // --- 1. calibration: noise scans -> W (strategy.rs:783-798) -------------
    bool have_w = false;
    int w_nc = 0;
    DevBuf dW(ctx), dWstat(ctx);
    if (cfg->prewhiten) {
        std::vector<long long> noise;
        for (long long a = 0; a < nacq; ++a)
            if (H[a].flags & ACQ_IS_NOISE_MEASUREMENT) noise.push_back(a);
        if (!noise.empty() && H[noise[0]].active_channels > 0) {
            const int nc = H[noise[0]].active_channels;
            long long total = 0, match = 0;
            for (long long a : noise) {
                total += H[a].number_of_samples;
                if (H[a].active_channels == nc) match += H[a].number_of_samples;
            }
            if (total >= nc && nc <= 128) {
                // concatenate the matching scans along samples: [nc][match]
                DevBuf dn(ctx);
                OKS_CUDA(dn.alloc(sizeof(float2) * (size_t)nc * (match ? match : 1)));
                long long col = 0;
                for (long long a : noise) {
                    if (H[a].active_channels != nc) continue;
                    const int ns = H[a].number_of_samples;
                    OKS_CUDA(cudaMemcpy2DAsync(dn.as<float2>() + col, sizeof(float2) * match,
                                               A->data + H[a].data_offset, sizeof(float2) * ns, sizeof(float2) * ns,
                                               nc, copy_kind, ctx->stream));
                    col += ns;
                }
                OKS_CUDA(dW.alloc(sizeof(float2) * (size_t)nc * nc));
                OKS_CUDA(dWstat.alloc(sizeof(int)));
                // no host round trip: a fit that fails (None, prewhiten.rs:161)
                // leaves its status word set and the apply kernel skips
                int rc = prewhiten_fit_launch(ctx, reinterpret_cast<const okscuda_c64*>(dn.p), nc, match, total,
                                              dW.as<okscuda_c64>(), dWstat.as<int>());
                if (rc == OKS_OK) { have_w = true; w_nc = nc; }
                else if (rc != OKS_ESKIP) return rc;
            }
        }
    }
    // --- 1b. calibration: navigator scans -> per-(slice, segment) phasors ----
    // (phasecorr.rs:61-129): bins in order of first appearance; a scan whose
    // sample count differs from its bin's first scan is dropped
    std::map<std::pair<int, int>, int> pc_bin_of;
    std::vector<oks::PcBin> pc_bins;
    DevBuf dnav(ctx), dcorr(ctx), dpct(ctx);   // navigators, phasors, bin + scan tables
    if (cfg->phase_correct) {
        std::vector<std::vector<long long>> members;
        for (long long a = 0; a < nacq; ++a) {
            if (!(H[a].flags & ACQ_IS_PHASECORR_DATA)) continue;
            const int ns = H[a].number_of_samples, anc = H[a].active_channels;
            if (ns == 0 || anc == 0) continue;
            const auto key = std::make_pair((int)H[a].slice, (int)H[a].segment);
            auto it = pc_bin_of.find(key);
            if (it == pc_bin_of.end()) {
                it = pc_bin_of.emplace(key, (int)pc_bins.size()).first;
                oks::PcBin b{};
                b.ns = ns;
                pc_bins.push_back(b);
                members.emplace_back();
            }
            if (pc_bins[it->second].ns != ns) continue;
            members[it->second].push_back(a);
        }
        if (!pc_bins.empty()) {
            std::vector<oks::PcScan> scans;
            long long nav_len = 0, corr_len = 0;
            int max_ns = 0;
            for (size_t b = 0; b < pc_bins.size(); ++b) {
                pc_bins[b].first = (int)scans.size();
                pc_bins[b].count = (int)members[b].size();
                pc_bins[b].corr = corr_len;
                corr_len += pc_bins[b].ns;
                max_ns = std::max(max_ns, pc_bins[b].ns);
                for (long long a : members[b]) {
                    oks::PcScan sc{};
                    sc.off = nav_len;
                    sc.nc = H[a].active_channels;
                    scans.push_back(sc);
                    nav_len += (long long)sc.nc * pc_bins[b].ns;
                }
            }
            OKS_CUDA(dnav.alloc(sizeof(float2) * (size_t)nav_len));
            OKS_CUDA(dcorr.alloc(sizeof(float2) * (size_t)corr_len));
            for (size_t b = 0; b < pc_bins.size(); ++b)
                for (size_t i = 0; i < members[b].size(); ++i) {
                    const okscuda_acq_header& h = H[members[b][i]];
                    OKS_CUDA(cudaMemcpyAsync(dnav.as<float2>() + scans[pc_bins[b].first + i].off, A->data + h.data_offset,
                                             sizeof(float2) * (size_t)h.active_channels * h.number_of_samples, copy_kind,
                                             ctx->stream));
                }
            // bins then scans, through a staging slot into memory this call owns
            std::vector<unsigned char> tab(sizeof(oks::PcBin) * pc_bins.size() + sizeof(oks::PcScan) * scans.size());
            std::memcpy(tab.data(), pc_bins.data(), sizeof(oks::PcBin) * pc_bins.size());
            std::memcpy(tab.data() + sizeof(oks::PcBin) * pc_bins.size(), scans.data(), sizeof(oks::PcScan) * scans.size());
            OKS_CUDA(dpct.alloc(tab.size()));
            oks::Staging::Slot* slot = nullptr;
            int rc = stage_upload(ctx, tab.data(), tab.size(), &slot);
            if (rc) return rc;
            OKS_CUDA(cudaMemcpyAsync(dpct.p, slot->dev, tab.size(), cudaMemcpyDeviceToDevice, ctx->stream));
            stage_release(ctx, slot);
            const auto* dbins = dpct.as<oks::PcBin>();
            const auto* dscans = reinterpret_cast<const oks::PcScan*>(dbins + pc_bins.size());
            ProfScope ps(ctx, "k_phasecorr_fit");
            OKS_CUDA(oks::launch_phasecorr_fit(dnav.as<float2>(), dscans, dbins, (int)pc_bins.size(), max_ns,
                                               dcorr.as<float2>(), ctx->stream));
        }
    }
    // bin of an image line: (slice, segment), else (u16::MAX, segment) (phasecorr.rs:145-153)
    auto pc_bin = [&](const okscuda_acq_header& h) {
        if (pc_bins.empty()) return -1;
        auto it = pc_bin_of.find({(int)h.slice, (int)h.segment});
        if (it == pc_bin_of.end()) it = pc_bin_of.find({65535, (int)h.segment});
        return it == pc_bin_of.end() ? -1 : it->second;
    };
    const bool os_on = cfg->remove_oversampling && os_ratio_ok(A->enc_x, A->rec_x);

    // --- 2. first pass over image scans: tensor shape (reader.rs:234-290) ----
    int max_ky = 0, max_kz = 0, max_slice = 0, max_samples = 0, nc_obs = 0;
    long long n_image = 0;
    bool three_d_seen = false;
    for (long long a = 0; a < nacq; ++a) {
        if (!is_image(H[a])) continue;
        ++n_image;
        max_ky = std::max<int>(max_ky, H[a].kspace_encode_step_1);
        max_kz = std::max<int>(max_kz, H[a].kspace_encode_step_2);
        max_slice = std::max<int>(max_slice, H[a].slice);
        max_samples = std::max<int>(max_samples, H[a].number_of_samples);
        nc_obs = std::max<int>(nc_obs, H[a].active_channels);
        if (H[a].kspace_encode_step_2 > 0) three_d_seen = true;   // reader.rs:187-202
    }
    if (n_image == 0) return set_err(ctx, OKS_EINVAL, "no image acquisitions found");
    if (nc_obs == 0) return set_err(ctx, OKS_EINVAL, "active_channels (0)");
    const bool use_slice_axis = max_kz == 0 && max_slice > 0;
    const int nx = std::max(A->enc_x, max_samples);
    const int ny = std::max(std::max(A->enc_y, max_ky + 1), 1);
    const int nz = use_slice_axis ? std::max(max_slice + 1, 1) : std::max(std::max(A->enc_z, max_kz + 1), 1);
    const int nc = nc_obs;
    const long long N = (long long)ny * nx;
    // output shape after maybe_crop (strategy.rs:227-253)
    int tz = nz, ty = ny, tx = nx;
    if (cfg->crop_to_recon_matrix) {
        const int cz = A->rec_z >= 2 ? std::min(A->rec_z, nz) : nz;
        const int cy = A->rec_y >= 1 ? std::min(A->rec_y, ny) : ny;
        const int cx = A->rec_x >= 1 ? std::min(A->rec_x, nx) : nx;
        if (cz != nz || cy != ny || cx != nx) { tz = cz; ty = cy; tx = cx; }
    }
    out_dims[0] = tz; out_dims[1] = ty; out_dims[2] = tx;
    const long long nout = (long long)tz * ty * tx;
    if (!h_out) return OKS_OK;   // shape query
    if (out_cap < nout) return set_err(ctx, OKS_EINVAL, "output buffer holds %lld floats, need %lld", out_cap, nout);

    // --- 3. second pass: preprocess + placement (reader.rs:332-457) ---------
    const int ky_off = ny / 2 - A->ky_center;
    const int kz_off = use_slice_axis ? 0 : nz / 2 - A->kz_center;
    std::vector<uint8_t>& filled = ctx->h_filled;   // kept across calls
    filled.assign((size_t)nz * N, 0);
    DevBuf dk(ctx);
    OKS_CUDA(dk.alloc(sizeof(float2) * (size_t)nc * nz * N));
    OKS_CUDA(cudaMemsetAsync(dk.p, 0, sizeof(float2) * (size_t)nc * nz * N, ctx->stream));
    // group image scans by (channels, samples) so each group is one batch
    std::map<std::pair<int, int>, std::vector<long long>> groups;
    for (long long a = 0; a < nacq; ++a)
        if (is_image(H[a])) groups[{H[a].active_channels, H[a].number_of_samples}].push_back(a);
    for (auto& g : groups) {
        const int gnc = g.first.first, gns = g.first.second;
        const std::vector<long long>& ids = g.second;
        if (gnc == 0 || gns == 0) continue;
        const long long ng = (long long)ids.size();
        DevBuf raw(ctx);
        OKS_CUDA(raw.alloc(sizeof(float2) * (size_t)ng * gnc * gns));
        // gather (contiguous runs are one copy)
        ProfScope ps_copy(ctx, A->data_on_device ? "copy_lines_d2d" : "copy_lines_h2d", nullptr, 0);   // no kernel
        for (long long i = 0; i < ng;) {
            long long j = i + 1;
            while (j < ng && H[ids[j]].data_offset == H[ids[j - 1]].data_offset + (long long)gnc * gns) ++j;
            OKS_CUDA(cudaMemcpyAsync(raw.as<float2>() + i * gnc * gns, A->data + H[ids[i]].data_offset,
                                     sizeof(float2) * (size_t)(j - i) * gnc * gns, copy_kind, ctx->stream));
            i = j;
        }
        // preprocess: W s (prewhiten.rs:118-124 skips other channel counts), then OS removal
        if (have_w && gnc == w_nc) {
            if (gnc > 64) return set_err(ctx, OKS_ENOTSUP, "prewhiten_apply: nc=%d above 64", gnc);
            if (ctx->prewhiten_bulk) {
                const int rc = tc_err_flag(ctx);
                if (rc) return rc;
            }
            ProfScope ps(ctx, oks::prewhiten_bulk_eligible(raw.as<float2>(), gnc, gns, ctx->tc_err,
                                                           ctx->prewhiten_bulk)
                                  ? "k_prewhiten_bulk"
                                  : "k_prewhiten_apply");
            OKS_CUDA(oks::launch_prewhiten_apply(raw.as<float2>(), dW.as<float2>(), ng, gnc, gns, ctx->stream,
                                                 dWstat.as<int>(), ctx->tc_err, ctx->prewhiten_bulk));
        }
        // navigator phasors (phasecorr.rs:141-168), before oversampling removal
        if (!pc_bins.empty()) {
            std::vector<int> sb(ng);
            bool any = false;
            for (long long i = 0; i < ng; ++i) {
                sb[i] = pc_bin(H[ids[i]]);
                any = any || sb[i] >= 0;
            }
            if (any) {
                oks::Staging::Slot* slot = nullptr;
                int rc = stage_upload(ctx, sb.data(), sizeof(int) * sb.size(), &slot);
                if (rc) return rc;
                cudaError_t e;
                {
                    ProfScope ps(ctx, "k_phasecorr_apply");
                    e = oks::launch_phasecorr_apply(raw.as<float2>(), ng, gnc, gns, static_cast<const int*>(slot->dev),
                                                    dpct.as<oks::PcBin>(), dcorr.as<float2>(),
                                                    ctx->stream);
                }
                stage_release(ctx, slot);
                if (e != cudaSuccess) return cuda_err(ctx, e, "phase correction");
            }
        }
        int pns = gns;
        DevBuf os(ctx);
        const float2* src = raw.as<float2>();
        const bool os_here = os_on && gns == A->enc_x;     // oversampling.rs:104-107
        if (os_here) {
            OKS_CUDA(os.alloc(sizeof(float2) * (size_t)ng * gnc * A->rec_x));
            int rc = okscuda_os_remove(ctx, raw.as<okscuda_c64>(), os.as<okscuda_c64>(), ng * gnc, A->enc_x, A->rec_x);
            if (rc) return rc;
            pns = A->rec_x;
            src = os.as<float2>();
        }
        // placement geometry (host), first wins
        std::vector<oks::PlaceEntry> tab;
        tab.reserve(ng);
        for (long long i = 0; i < ng; ++i) {
            const okscuda_acq_header& h = H[ids[i]];
            const int ky = (int)h.kspace_encode_step_1 + ky_off;
            const int kz = (use_slice_axis ? (int)h.slice : (int)h.kspace_encode_step_2) + kz_off;
            if (ky < 0 || ky >= ny || kz < 0 || kz >= nz) continue;
            // oversampling.rs:147-153 rewrites the header of a processed line
            const size_t ns = pns;
            const size_t dpre = os_here ? 0 : h.discard_pre, dpost = os_here ? 0 : h.discard_post;
            const size_t cs = os_here ? (size_t)(A->rec_x / 2) : h.center_sample;
            const size_t keep = sat_sub(ns, dpre + dpost);
            const size_t dst = (cs > 0 && cs >= dpre) ? sat_sub((size_t)nx / 2, cs - dpre) : sat_sub(nx, keep) / 2;
            const size_t src_len = std::min(keep, sat_sub(ns, dpre));
            const size_t len = std::min(src_len, sat_sub(nx, dst));
            if (len == 0) continue;
            const size_t centre = dst + len / 2;
            uint8_t* frow = filled.data() + ((size_t)kz * ny + ky) * nx;
            if (frow[centre]) continue;
            std::memset(frow + dst, 1, len);
            oks::PlaceEntry e{};
            e.acq = i; e.kz = kz; e.ky = ky; e.dst_off = (int)dst; e.src_off = (int)dpre; e.len = (int)len;
            e.reverse = (h.flags & ACQ_IS_REVERSE) ? 1 : 0;
            e.nc_fit = std::min(gnc, nc);
            tab.push_back(e);
        }
        if (!tab.empty()) {
            oks::Staging::Slot* slot = nullptr;
            int rc = stage_upload(ctx, tab.data(), tab.size() * sizeof(oks::PlaceEntry), &slot);
            if (rc) return rc;
            cudaError_t e;
            {
                ProfScope ps(ctx, "k_place");
                e = oks::launch_place(src, gnc, pns, static_cast<const oks::PlaceEntry*>(slot->dev),
                                      (long long)tab.size(), dk.as<float2>(), nz, ny, nx, ctx->stream);
            }
            stage_release(ctx, slot);
            if (e != cudaSuccess) return cuda_err(ctx, e, "placement");
        }
    }

    // --- 4. 3-D decoupling (strategy.rs:817-827) ----------------------------
    const bool three_d = cfg->fft_mode == 2 || (cfg->fft_mode == 0 && three_d_seen);
    if (three_d) {
        int rc = okscuda_ifft1_kz(ctx, dk.as<okscuda_c64>(), nc, nz, ny, nx);
        if (rc) return rc;
    }
    const int z0 = (nz - tz) / 2;

    DevBuf coils(ctx), rss(ctx);
    OKS_CUDA(rss.alloc(sizeof(float) * (size_t)nout));
    if (ny % 2 || nx % 2) {
        // --- 6. odd dims: IFFT + RSS fallback (strategy.rs:829-842) ----------
        int rc = okscuda_ifft2(ctx, dk.as<okscuda_c64>(), (long long)nc * nz, ny, nx);
        if (rc) return rc;
    } else {
        // --- 7. per-slice per-coil FISTA (strategy.rs:849-869) -----------------
        int rc = oks_fista_core(ctx, dk.as<okscuda_c64>(), filled.data(), nz, (long long)nc * nz, ny, nx, cfg->iters,
                                cfg->lambda, dk.as<okscuda_c64>());
        if (rc) return rc;
    }
    // --- 8. RSS (strategy.rs:870-879) + crop ---------------------------------
    oks::RssArgs ra{};
    ra.coils = dk.as<float2>() + (long long)z0 * N;
    ra.coil_stride = (long long)nz * N;
    ra.nc = nc; ra.ny = ny; ra.nx = nx;
    ra.nslice = tz; ra.slice_stride = N;
    ra.ty = ty; ra.tx = tx; ra.y0 = (ny - ty) / 2; ra.x0 = (nx - tx) / 2;
    ra.out = rss.as<float>();
    {
        ProfScope ps(ctx, "k_rss");
        OKS_CUDA(oks::launch_rss(ra, ctx->stream));
    }
    // device-resident mode (data_on_device): h_out is a device buffer and the
    // call returns without waiting
    {
        ProfScope ps(ctx, A->data_on_device ? "copy_out_d2d" : "copy_out_d2h", nullptr, 0);   // no kernel
        OKS_CUDA(cudaMemcpyAsync(h_out, rss.p, sizeof(float) * (size_t)nout,
                                 A->data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (!A->data_on_device) OKS_CUDA(cudaStreamSynchronize(ctx->stream));
    return OKS_OK;
}

}  // extern "C"
