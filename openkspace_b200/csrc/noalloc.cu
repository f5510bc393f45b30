// okscuda_cs_slice_noalloc: the per-slice FISTA-CS + RSS of okscuda_cs_slice
// for callers that cannot allocate device memory -- applications that hand
// all device memory to their own allocator (a framework memory pool, or a
// scanner pipeline that reserves its budget at start-up and forbids device
// allocation afterwards).  No device or pinned host memory is allocated: the
// coil images, FFT tables (those of the register row transform included),
// momentum weights and row mask live in one file-scope device array,
// `g_noalloc_scratch`, which every GPU that loads this library holds until
// the process exits.
//
// Host code never uses the array's name as an address: in host code it is a
// host-side stand-in, and a kernel given it would fault (or, where the GPU
// can reach host memory, quietly use the wrong memory).  The first call on
// each device looks the real device address up with cudaGetSymbolAddress
// while that device is current, checks the return code and caches it; make
// that first call before any stream capture.
//
// Every call shares the array and it keeps the last call's contents.  Each
// call rewrites every byte it reads before reading it, so nothing needs
// clearing, but calls that overlap on the GPU (other streams, other contexts
// on the same device) race on it: serialise them.
#include <mutex>

#include "ctx.h"

namespace {

constexpr size_t kNoAllocBytes = 16u << 20;          // 16 MiB in total
constexpr size_t kTableBytes = 256u << 10;           // FFT tables, weights, mask
constexpr size_t kDataBytes = kNoAllocBytes - kTableBytes;
constexpr int kMaxN = 2048;                          // ny, nx limit of this entry point
constexpr int kMaxIters = 8192;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_mu;
void* g_dev_addr[64] = {};                           // per-device address of the array
unsigned char g_host_tables[kTableBytes];            // host staging of the table region

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" int okscuda_cs_slice_noalloc(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask,
                                        int nc, int ny, int nx, int iters, float lambda, float* d_rss) {
    OKS_CHECK_CTX();
    if (!d_kspace || !h_mask || !d_rss || nc <= 0 || ny <= 0 || nx <= 0 || iters < 0)
        return set_err(ctx, OKS_EINVAL, "cs_slice_noalloc: bad arguments");
    if (ny % 2 || nx % 2)
        return set_err(ctx, OKS_EODD, "CS: Ny (%d) and Nx (%d) must both be even for Haar wavelet", ny, nx);
    const size_t data_bytes = sizeof(float2) * (size_t)nc * ny * nx;
    if (ny > kMaxN || nx > kMaxN || iters > kMaxIters || data_bytes > kDataBytes)
        return set_err(ctx, OKS_ENOTSUP,
                       "cs_slice_noalloc: nc*ny*nx*8 = %zu bytes exceeds the fixed %zu-byte scratch "
                       "(or ny, nx > %d, or iters > %d); use okscuda_cs_slice",
                       data_bytes, kDataBytes, kMaxN, kMaxIters);
    int dev = ctx->device;
    if (dev < 0 || dev >= 64) return set_err(ctx, OKS_ENOTSUP, "cs_slice_noalloc: device %d", dev);

    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // this device is current
        if (e != cudaSuccess || !p) return cuda_err(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_dev_addr[dev] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(g_dev_addr[dev]);

    // ky-only mask as row bits (the 2-D engine needs more scratch than this array)
    const int wstride = (ny + 31) / 32;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    const size_t o_mask = take(sizeof(uint32_t) * wstride);
    const size_t o_alpha = take(sizeof(float) * (iters > 0 ? iters : 1));
    const size_t o_twy = take(sizeof(float2) * (2 * ny + 1));
    const size_t o_rty = take(sizeof(float2) * (ny + 1));
    const size_t o_twx = take(sizeof(float2) * (2 * nx + 1));
    const size_t o_rtx = take(sizeof(float2) * (nx + 1));
    constexpr int kRegTab = 4096 + 64;                // register row plan: twiddles + roots
    const size_t o_reg = take(sizeof(float2) * kRegTab);
    if (off > kTableBytes) return set_err(ctx, OKS_ENOTSUP, "cs_slice_noalloc: tables exceed %zu bytes", kTableBytes);

    uint32_t* words = reinterpret_cast<uint32_t*>(g_host_tables + o_mask);
    for (int w = 0; w < wstride; ++w) words[w] = 0u;
    for (int r = 0; r < ny; ++r) {
        const uint8_t* m = h_mask + (size_t)r * nx;
        const bool on = m[0] != 0;
        for (int x = 1; x < nx; ++x)
            if ((m[x] != 0) != on)
                return set_err(ctx, OKS_ENOTSUP, "cs_slice_noalloc: mask varies along kx (use okscuda_cs_slice)");
        if (on) words[r >> 5] |= 1u << (r & 31);
    }
    float* alpha = reinterpret_cast<float*>(g_host_tables + o_alpha);   // cs.rs:125-126 in f32
    float t = 1.0f;
    for (int i = 0; i < iters; ++i) {
        const float t_new = 0.5f * (1.0f + std::sqrt(1.0f + 4.0f * t * t));
        alpha[i] = (t - 1.0f) / t_new;
        t = t_new;
    }
    oks::DevPlan py, px;
    int ntw, nrt;
    if (!oks::build_plan_into(ny, &py.plan, reinterpret_cast<float2*>(g_host_tables + o_twy), 2 * ny + 1, &ntw,
                              reinterpret_cast<float2*>(g_host_tables + o_rty), ny + 1, &nrt))
        return set_err(ctx, OKS_ENOTSUP, "cs_slice_noalloc: no FFT plan for ny=%d", ny);
    py.roots_total = nrt;
    if (!oks::build_plan_into(nx, &px.plan, reinterpret_cast<float2*>(g_host_tables + o_twx), 2 * nx + 1, &ntw,
                              reinterpret_cast<float2*>(g_host_tables + o_rtx), nx + 1, &nrt))
        return set_err(ctx, OKS_ENOTSUP, "cs_slice_noalloc: no FFT plan for nx=%d", nx);
    px.roots_total = nrt;
    py.tw = reinterpret_cast<float2*>(base + o_twy);
    py.roots = reinterpret_cast<float2*>(base + o_rty);
    px.tw = reinterpret_cast<float2*>(base + o_twx);
    px.roots = reinterpret_cast<float2*>(base + o_rtx);
    // the register row transform's tables go into the array too (the
    // library's own per-length tables would be allocated on first use)
    int reg_nroots = 0;
    const int reg_n = ctx->xform_reg && oks::xform_reg_supported(nx)
                          ? oks::row_xform_reg_tables(nx, reinterpret_cast<float2*>(g_host_tables + o_reg), kRegTab,
                                                      &reg_nroots)
                          : 0;
    // pageable source: returns once the bytes are staged, so the host tables
    // may be rewritten by the next call
    OKS_CUDA(cudaMemcpyAsync(base, g_host_tables, off, cudaMemcpyHostToDevice, ctx->stream));

    float2* coils = reinterpret_cast<float2*>(base + kTableBytes);
    const oks::RowMasks rm{reinterpret_cast<const uint32_t*>(base + o_mask), wstride, 1};
    oks::RowXformArgs ra{};
    ra.reg = reg_n > 0 ? 1 : 0;
    ra.tables = reg_n > 0 ? reinterpret_cast<const float2*>(base + o_reg) : nullptr;
    ra.tables_nroots = reg_nroots;
    ra.in = reinterpret_cast<const float2*>(d_kspace);
    ra.out = coils;
    ra.nrows = (long long)nc * ny;
    ra.ld_in = nx; ra.ld_out = nx;
    ra.sign = +1; ra.centred = 1;
    ra.scale = std::sqrt((float)ny) / std::sqrt((float)nx) * (((ny / 2) & 1) ? -1.0f : 1.0f);
    ra.rows_per_prob = ny; ra.rowsign = 1;
    ra.use_keep = 1; ra.keep = rm;
    OKS_CUDA(oks::launch_row_xform(ra, px, ctx->stream));
    oks::FistaColArgs fa{};
    fa.ytil = coils; fa.prob_stride = (long long)ny * nx;
    fa.minv = 1.0f / (float)ny;
    fa.mask = rm;
    fa.xout = coils; fa.out_stride = (long long)ny * nx;
    fa.ny = ny; fa.nx = nx; fa.iters = iters; fa.lambda = lambda;
    fa.alpha = reinterpret_cast<const float*>(base + o_alpha);
    fa.nprob = nc;
    OKS_CUDA(oks::launch_fista_col(fa, py, ctx->stream));
    oks::RssArgs rs{};
    rs.coils = coils; rs.coil_stride = (long long)ny * nx;
    rs.nc = nc; rs.ny = ny; rs.nx = nx;
    rs.nslice = 1; rs.slice_stride = 0;
    rs.ty = ny; rs.tx = nx; rs.y0 = 0; rs.x0 = 0;
    rs.out = d_rss;
    OKS_CUDA(oks::launch_rss(rs, ctx->stream));
    return OKS_OK;
}
