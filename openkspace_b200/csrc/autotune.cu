// Autotuner for the FISTA engines' plans and launch shapes (no reference
// counterpart: the reference has one CPU code path).  For one shape it
// times every candidate on seeded synthetic k-space made on the device, then
// keeps the fastest in the context's per-shape table, which the engines
// consult at dispatch (ctx.h tune_params).
//   kind 0, ky-only masks (column engine): register kernel with the primary
//            plan, with the E = 8 alternative plan where one exists, and the
//            generic shared-memory kernel;
//   kind 1, 2-D masks (partial rows, as after readout-oversampling removal):
//            register budgets, pipelined column loads, persistent grids,
//            chunks in flight and chunk sizes of the two-pass engine.
// The table can be read out as text and loaded back (okscuda_autotune_table /
// okscuda_autotune_load), so a deployment tunes once per GPU model.
#include <sstream>

#include "ctx.h"

namespace {

__global__ void k_fill_random(float2* d, long long n, unsigned seed) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        // integer hash (splitmix-style) of (seed, i) to two uniforms in [-1, 1)
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        d[i] = make_float2((float)(z & 0xFFFFFFu) / 8388608.f - 1.f, (float)((z >> 24) & 0xFFFFFFu) / 8388608.f - 1.f);
    }
}

std::string describe(const TuneParams& p) {
    std::ostringstream o;
    o << "col_engine=" << p.col_engine << " col_variant=" << p.col_variant << " persist2d=" << p.persist2d
      << " occ2d=" << p.occ2d << " prefetch2d=" << p.prefetch2d << " fista2d_streams=" << p.fista2d_streams
      << " fista2d_chunk=" << p.fista2d_chunk;
    return o.str();
}

}  // namespace

extern "C" int okscuda_autotune(okscuda_ctx* ctx, int kind, int ny, int nx, int nc, int iters, char* report,
                                size_t report_len) {
    OKS_CHECK_CTX();
    if ((kind != 0 && kind != 1) || ny <= 0 || nx <= 0 || nc <= 0 || iters <= 0 || ny % 2 || nx % 2 ||
        (kind == 1 && nx < 8))
        return set_err(ctx, OKS_EINVAL, "autotune: bad arguments");
    const long long N = (long long)ny * nx;
    // ky mask: every 4th row plus an 8 % centre; kind 1 keeps only the
    // central half of kx on the sampled rows
    std::vector<uint8_t> mask((size_t)N, 0);
    const int c0 = ny / 2 - std::max(1, ny / 25), c1 = ny / 2 + std::max(1, ny / 25);
    for (int r = 0; r < ny; ++r) {
        if (!(r % 4 == 1 || (r >= c0 && r < c1))) continue;
        for (int x = 0; x < nx; ++x)
            if (kind == 0 || (x >= nx / 4 && x < nx / 4 + nx / 2)) mask[(size_t)r * nx + x] = 1;
    }
    float2* d = nullptr;
    OKS_CUDA(cudaMallocAsync(&d, sizeof(float2) * 2 * nc * N, ctx->stream));
    float2* out = d + nc * N;
    k_fill_random<<<148 * 4, 256, 0, ctx->stream>>>(d, nc * N, 12345u);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { cudaFreeAsync(d, ctx->stream); return cuda_err(ctx, e, "autotune data"); }

    TuneParams base{ctx->col_engine, ctx->col_variant < 0 ? 0 : ctx->col_variant, ctx->persist2d, ctx->occ2d,
                    ctx->prefetch2d, ctx->fista2d_streams, ctx->fista2d_chunk};
    std::vector<TuneParams> cands;
    if (kind == 0) {
        TuneParams p = base;
        p.col_engine = 2; p.col_variant = 0;
        if (oks::fista_col_reg_supported(ny)) cands.push_back(p);
        if (oks::fista_col_reg_variants(ny) > 1) { p.col_variant = 1; cands.push_back(p); }
        p.col_engine = 1; p.col_variant = 0;
        cands.push_back(p);
    } else {
        const long long autochunk = std::max<long long>(1, (96ll << 20) / (4 * N * 8));
        const int chunk_mult[3] = {1, 2, 0};   // x1, x1/2, x1.5 (0 encodes 3/2)
        for (int occ : {1, 0, 2})
            for (int pf : {1, 0, 3})
                for (int ns : {2, 3, 1})
                    for (int cm : chunk_mult) {
                        TuneParams p = base;
                        p.col_engine = 0;
                        p.persist2d = 1;
                        p.occ2d = occ;
                        p.prefetch2d = pf;
                        p.fista2d_streams = ns;
                        p.fista2d_chunk = cm == 1 ? autochunk : cm == 2 ? std::max(1ll, autochunk / 2)
                                                                         : autochunk * 3 / 2;
                        // a pruned grid: vary one or two knobs around the default
                        const int changed = (occ != 1) + (pf != 1) + (ns != 2) + (cm != 1);
                        if (changed <= 1 || (changed == 2 && cm != 1 && ns != 2)) cands.push_back(p);
                    }
    }
    const auto key = std::make_tuple(kind, ny, kind == 0 ? 0 : nx);
    const int saved_use = ctx->use_tuned;
    auto saved = ctx->tuned;
    std::ostringstream rep;
    rep << "{\"kind\": " << kind << ", \"ny\": " << ny << ", \"nx\": " << nx << ", \"nc\": " << nc
        << ", \"iters\": " << iters << ", \"candidates\": [";
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int rc = OKS_OK;
    if ((e = cudaEventCreate(&ev0)) != cudaSuccess || (e = cudaEventCreate(&ev1)) != cudaSuccess)
        rc = cuda_err(ctx, e, "autotune events");
    float best_ms = 1e30f;
    int best = -1;
    for (size_t i = 0; i < cands.size() && !rc; ++i) {
        ctx->tuned[key] = cands[i];
        ctx->use_tuned = 1;
        // one untimed call (plans, tables, pools), then the best of two
        rc = oks_fista_core(ctx, reinterpret_cast<okscuda_c64*>(d), mask.data(), 1, nc, ny, nx, iters, 0.01f,
                            reinterpret_cast<okscuda_c64*>(out));
        float ms = 1e30f;
        for (int rep_i = 0; rep_i < 2 && !rc; ++rep_i) {
            cudaEventRecord(ev0, ctx->stream);
            rc = oks_fista_core(ctx, reinterpret_cast<okscuda_c64*>(d), mask.data(), 1, nc, ny, nx, iters, 0.01f,
                                reinterpret_cast<okscuda_c64*>(out));
            cudaEventRecord(ev1, ctx->stream);
            if ((e = cudaEventSynchronize(ev1)) != cudaSuccess) { rc = cuda_err(ctx, e, "autotune timing"); break; }
            float t = 0.f;
            cudaEventElapsedTime(&t, ev0, ev1);
            ms = std::min(ms, t);
        }
        if (rc) break;
        rep << (i ? ", " : "") << "{\"params\": \"" << describe(cands[i]) << "\", \"ms\": " << ms << "}";
        if (ms < best_ms) { best_ms = ms; best = (int)i; }
    }
    ctx->tuned = saved;
    ctx->use_tuned = saved_use;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    cudaFreeAsync(d, ctx->stream);
    if (rc) return rc;
    if (best < 0) return set_err(ctx, OKS_ENOTSUP, "autotune: no candidate for this shape");
    ctx->tuned[key] = cands[best];
    rep << "], \"chosen\": \"" << describe(cands[best]) << "\", \"ms\": " << best_ms << "}";
    if (report && report_len) std::snprintf(report, report_len, "%s", rep.str().c_str());
    return OKS_OK;
}

// One line per tuned shape: kind ny nx col_engine col_variant persist2d occ2d
// prefetch2d fista2d_streams fista2d_chunk.
extern "C" int okscuda_autotune_table(okscuda_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || !len) return OKS_EINVAL;
    std::ostringstream o;
    for (const auto& kv : ctx->tuned) {
        const TuneParams& p = kv.second;
        o << std::get<0>(kv.first) << " " << std::get<1>(kv.first) << " " << std::get<2>(kv.first) << " "
          << p.col_engine << " " << p.col_variant << " " << p.persist2d << " " << p.occ2d << " " << p.prefetch2d
          << " " << p.fista2d_streams << " " << p.fista2d_chunk << "\n";
    }
    const std::string s = o.str();
    if (s.size() + 1 > len) return set_err(ctx, OKS_EINVAL, "autotune_table: buffer of %zu bytes too small", len);
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return OKS_OK;
}

extern "C" int okscuda_autotune_load(okscuda_ctx* ctx, const char* text) {
    if (!ctx || !text) return OKS_EINVAL;
    std::istringstream in(text);
    std::string line;
    std::map<std::tuple<int, int, int>, TuneParams> add;
    while (std::getline(in, line)) {
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        std::istringstream ls(line);
        int kind, ny, nx;
        TuneParams p{};
        if (!(ls >> kind >> ny >> nx >> p.col_engine >> p.col_variant >> p.persist2d >> p.occ2d >> p.prefetch2d >>
              p.fista2d_streams >> p.fista2d_chunk) ||
            (kind != 0 && kind != 1) || ny <= 0 || nx < 0 || p.col_engine < 0 || p.col_engine > 2 ||
            p.col_variant < 0 || p.col_variant > 1 || p.prefetch2d < 0 || p.prefetch2d > 3 ||
            p.fista2d_streams < 1 || p.fista2d_streams > 8 || p.fista2d_chunk < 0)
            return set_err(ctx, OKS_EINVAL, "autotune_load: bad line '%s'", line.c_str());
        add[std::make_tuple(kind, ny, kind == 0 ? 0 : nx)] = p;
    }
    for (auto& kv : add) ctx->tuned[kv.first] = kv.second;
    return OKS_OK;
}
