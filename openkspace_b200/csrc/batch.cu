// okscuda_cs_batch: many slices of uneven size, coil count, iteration count,
// lambda and mask in one batched pass (strategy.rs:850-880 applied to a list
// of independent slices).  Per column length there is one launch of the
// register-resident column engine whose units ((coil, column pair) of every
// slice) are ordered longest-first; the length groups run concurrently on
// forked streams.  Slices the batched engine cannot take (masks that vary
// along kx, column lengths without a compile-time plan) go through the
// per-slice path.
#include "ctx.h"

namespace {

struct Item {
    int req;
    int coil;
};

}  // namespace

// The batched pass on the context stream.  The column-length groups run on
// forked streams: aux[k % naux] (joined back before the RSS), the context's
// own auxiliary streams when aux is null.  The request server gives each of
// its batch slots separate fork streams, so that batches overlap.
int oks_cs_batch_core(okscuda_ctx* ctx, const okscuda_slice_req* reqs, int n, okscuda_ctx::Aux* aux, int naux,
                      cudaEvent_t fork_ev) {
    if (n < 0 || (n > 0 && !reqs)) return set_err(ctx, OKS_EINVAL, "cs_batch: bad arguments");
    if (n == 0) return OKS_OK;
    int max_iters = 0, wstride = 1;
    size_t scratch_elems = 0;
    for (int i = 0; i < n; ++i) {
        const okscuda_slice_req& r = reqs[i];
        if (!r.d_kspace || !r.h_mask || !r.d_rss || r.nc <= 0 || r.ny <= 0 || r.nx <= 0 || r.iters < 0)
            return set_err(ctx, OKS_EINVAL, "cs_batch: request %d has bad arguments", i);
        if (r.ny % 2 || r.nx % 2)
            return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", r.ny, r.nx);
        max_iters = std::max(max_iters, r.iters);
        wstride = std::max(wstride, (r.ny + 31) / 32);
        if (!r.d_coils) scratch_elems += (size_t)r.nc * r.ny * r.nx;
    }
    // row masks of every request; requests with masks that vary along kx or
    // without a register plan take the per-slice path
    std::vector<uint32_t> words((size_t)n * wstride, 0u);
    std::vector<char> batched(n, 0);
    for (int i = 0; i < n; ++i) {
        const okscuda_slice_req& r = reqs[i];
        bool sep = true;
        for (int y = 0; y < r.ny && sep; ++y) {
            const uint8_t* m = r.h_mask + (size_t)y * r.nx;
            const bool on = m[0] != 0;
            for (int x = 1; x < r.nx; ++x)
                if ((m[x] != 0) != on) { sep = false; break; }
            if (on) words[(size_t)i * wstride + (y >> 5)] |= 1u << (y & 31);
        }
        batched[i] = sep && oks::fista_col_reg_supported(r.ny) && tune_params(ctx, 0, r.ny, 0).col_engine != 1;
    }
    void* scratch = nullptr;
    if (scratch_elems) OKS_CUDA(cudaMallocAsync(&scratch, sizeof(float2) * scratch_elems, ctx->stream));
    std::vector<float2*> coils(n);
    {
        size_t o = 0;
        for (int i = 0; i < n; ++i) {
            if (reqs[i].d_coils) coils[i] = reinterpret_cast<float2*>(reqs[i].d_coils);
            else { coils[i] = static_cast<float2*>(scratch) + o; o += (size_t)reqs[i].nc * reqs[i].ny * reqs[i].nx; }
        }
    }
    int rc = OKS_OK;
    cudaError_t e = cudaSuccess;
    oks::Staging::Slot* mslot = nullptr;
    const float* alpha = nullptr;
    rc = get_alpha(ctx, std::max(max_iters, 1), &alpha);
    if (!rc) rc = stage_upload(ctx, words.data(), words.size() * sizeof(uint32_t), &mslot);
    if (!rc) e = oks::reg_tables_init(&ctx->reg_tables);
    if (!rc && e != cudaSuccess) rc = cuda_err(ctx, e, "register tables");
    const uint32_t* dwords = mslot ? static_cast<const uint32_t*>(mslot->dev) : nullptr;

    // 1. y' for every batched request (row IDFT of the masked k-space)
    for (int i = 0; i < n && !rc; ++i) {
        if (!batched[i]) continue;
        const okscuda_slice_req& r = reqs[i];
        const DevPlan* px;
        if ((rc = get_plan(ctx, r.nx, &px))) break;
        oks::RowXformArgs ra{};
        ra.reg = ctx->xform_reg;
        ra.in = reinterpret_cast<const float2*>(r.d_kspace);
        ra.out = coils[i];
        ra.nrows = (long long)r.nc * r.ny;
        ra.ld_in = r.nx; ra.ld_out = r.nx;
        ra.sign = +1; ra.centred = 1;
        ra.scale = std::sqrt((float)r.ny) / std::sqrt((float)r.nx) * (((r.ny / 2) & 1) ? -1.0f : 1.0f);
        ra.rows_per_prob = r.ny; ra.rowsign = 1;
        ra.use_keep = 1;
        ra.keep = oks::RowMasks{dwords + (size_t)i * wstride, wstride, 1};
        ProfScope ps(ctx, "k_row_xform");
        if ((e = oks::launch_row_xform(ra, *px, ctx->stream)) != cudaSuccess) rc = cuda_err(ctx, e, "row pass");
    }
    // 2. one register-engine launch per column length, longest units first
    std::map<int, std::vector<Item>> groups;
    for (int i = 0; i < n; ++i)
        if (batched[i])
            for (int c = 0; c < reqs[i].nc; ++c) groups[reqs[i].ny].push_back({i, c});
    std::vector<oks::ColProblem> table;
    std::vector<std::pair<size_t, size_t>> spans;   // [begin, end) of each group in `table`
    std::vector<long long> nunits;
    for (auto& g : groups) {
        auto& items = g.second;
        std::stable_sort(items.begin(), items.end(), [&](const Item& a, const Item& b) {
            return (long long)reqs[a.req].iters * reqs[a.req].ny > (long long)reqs[b.req].iters * reqs[b.req].ny;
        });
        const size_t begin = table.size();
        long long u = 0;
        for (const Item& it : items) {
            const okscuda_slice_req& r = reqs[it.req];
            oks::ColProblem p{};
            p.y = coils[it.req] + (size_t)it.coil * r.ny * r.nx;
            p.x = const_cast<float2*>(p.y);
            p.nx = r.nx;
            p.iters = r.iters;
            p.lambda = r.lambda;
            p.mask = it.req;
            p.unit0 = u;
            u += r.nx / 2;
            table.push_back(p);
        }
        spans.push_back({begin, table.size()});
        nunits.push_back(u);
    }
    oks::Staging::Slot* tslot = nullptr;
    if (!rc && !table.empty()) rc = stage_upload(ctx, table.data(), table.size() * sizeof(oks::ColProblem), &tslot);
    if (!rc && !table.empty()) {
        // fork: group k on aux stream k (ordered after everything so far)
        const int ng = (int)spans.size();
        if (!aux) {
            rc = ensure_aux_streams(ctx, ng);
            aux = ctx->aux.data();
            naux = ng;
            fork_ev = ctx->fork_ev;
        }
        if (!rc) OKS_CUDA(cudaEventRecord(fork_ev, ctx->stream));
        int k = 0;
        for (auto& g : groups) {
            if (rc) break;
            okscuda_ctx::Aux& ax = aux[k % naux];
            cudaStream_t s = ax.stream;
            OKS_CUDA(cudaStreamWaitEvent(s, fork_ev, 0));
            oks::FistaColArgs fa{};
            fa.ny = g.first;
            fa.minv = 1.0f / (float)g.first;
            fa.mask = oks::RowMasks{dwords, wstride, n};
            fa.alpha = alpha;
            fa.probs = static_cast<const oks::ColProblem*>(tslot->dev) + spans[k].first;
            fa.nprob = (long long)(spans[k].second - spans[k].first);
            fa.nunits = nunits[k];
            fa.variant = tune_params(ctx, 0, g.first, 0).col_variant;
            fa.nx = 2;   // unused in the batched form; keeps the launch guard open
            {
                ProfScope ps(ctx, "k_fista_col_reg", s);
                e = oks::launch_fista_col_reg(fa, ctx->reg_tables, s);
            }
            if (e != cudaSuccess) rc = cuda_err(ctx, e, "batched column engine");
            OKS_CUDA(cudaEventRecord(ax.done, s));
            OKS_CUDA(cudaStreamWaitEvent(ctx->stream, ax.done, 0));
            ++k;
        }
    }
    // 3. requests outside the batched engine, one by one
    for (int i = 0; i < n && !rc; ++i) {
        if (batched[i]) continue;
        const okscuda_slice_req& r = reqs[i];
        rc = oks_fista_core(ctx, r.d_kspace, r.h_mask, 1, r.nc, r.ny, r.nx, r.iters, r.lambda,
                            reinterpret_cast<okscuda_c64*>(coils[i]));
    }
    // 4. RSS of every request (strategy.rs:870-879)
    for (int i = 0; i < n && !rc; ++i) {
        const okscuda_slice_req& r = reqs[i];
        oks::RssArgs a{};
        a.coils = coils[i];
        a.coil_stride = (long long)r.ny * r.nx;
        a.nc = r.nc; a.ny = r.ny; a.nx = r.nx;
        a.nslice = 1; a.slice_stride = 0;
        a.ty = r.ny; a.tx = r.nx; a.y0 = 0; a.x0 = 0;
        a.out = r.d_rss;
        ProfScope ps(ctx, "k_rss");
        if ((e = oks::launch_rss(a, ctx->stream)) != cudaSuccess) rc = cuda_err(ctx, e, "rss");
    }
    if (tslot) stage_release(ctx, tslot);
    if (mslot) stage_release(ctx, mslot);
    if (scratch) cudaFreeAsync(scratch, ctx->stream);
    return rc;
}

extern "C" int okscuda_cs_batch(okscuda_ctx* ctx, const okscuda_slice_req* reqs, int n) {
    OKS_CHECK_CTX();
    return oks_cs_batch_core(ctx, reqs, n, nullptr, 0, nullptr);
}
