// Output writers of the reconstruction (openkspace-cli/src/main.rs:1033-1153):
// percentile windowing to 8-bit on the device, NIfTI-1 and 8-bit PNG files on
// the host.
//
// * okscuda_percentile: main.rs:1147-1153 picks element round(pct/100 (n-1))
//   of the ascending sort.  Here that order statistic comes from a radix
//   select over the device array instead of a sort: float bits are mapped to
//   keys whose unsigned order is the float order, four 8-bit passes each
//   histogram the keys that still match the selected prefix and pick the bin
//   holding the wanted rank (a one-thread kernel, so the passes need no host
//   round trip).  The result is the exact element, bit for bit.
// * okscuda_window_u8: main.rs:1095-1140 per pixel, f32 arithmetic in the
//   reference's order: norm = clamp((v - lo) / (hi - lo), 0, 1), then
//   round(norm^0.9 * 255) (windowed) or round(norm * 255) (linear).
// * okscuda_write_nifti / okscuda_write_png: host files.  The NIfTI-1 header
//   follows main.rs:1033-1074 field by field (it is a file format); the PNG is
//   an 8-bit grayscale image whose zlib stream uses stored (uncompressed)
//   deflate blocks.
#include <cfloat>
#include <cstdio>

#include "ctx.h"

namespace oks {
namespace {

// Unsigned key with the order of the float: negative values reversed below
// the positive ones.  NaNs (positive or negative) map above +inf.
__device__ __forceinline__ uint32_t float_key(float f) {
    uint32_t u = __float_as_uint(f);
    if (f != f) return 0xFFFFFFFFu;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Select state: keys matching `prefix` on the bits of `mask` are candidates;
// `rank` is the wanted rank among them.
struct SelectState {
    uint32_t prefix;
    uint32_t mask;
    unsigned long long rank;
    unsigned long long hist[256];
};

__global__ void k_select_hist(const float* __restrict__ v, long long n, SelectState* st, int shift) {
    __shared__ unsigned int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t prefix = st->prefix, mask = st->mask;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t k = float_key(__ldg(v + i));
        if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&st->hist[i], (unsigned long long)h[i]);
}

// One thread: the bin that holds the wanted rank extends the prefix; the
// histogram is cleared for the next pass.
__global__ void k_select_pick(SelectState* st, int shift) {
    unsigned long long r = st->rank;
    int bin = 255;
    for (int b = 0; b < 256; ++b) {
        const unsigned long long c = st->hist[b];
        if (r < c) {
            bin = b;
            break;
        }
        r -= c;
    }
    st->rank = r;
    st->prefix |= (uint32_t)bin << shift;
    st->mask |= 255u << shift;
    for (int b = 0; b < 256; ++b) st->hist[b] = 0;
}

__global__ void k_window_u8(const float* __restrict__ v, long long n, float lo, float hi, int gamma,
                            uint8_t* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float norm = (__ldg(v + i) - lo) / (hi - lo);
        norm = fminf(fmaxf(norm, 0.0f), 1.0f);
        if (!(norm == norm)) {   // NaN casts to 0 (Rust `as u8`)
            out[i] = 0;
            continue;
        }
        const float g = gamma ? powf(norm, 0.9f) : norm;
        out[i] = (uint8_t)roundf(g * 255.0f);
    }
}

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 255u] ^ (crc >> 8);
    return ~crc;
}

void put_be32(std::vector<uint8_t>& b, uint32_t v) {
    b.push_back((uint8_t)(v >> 24));
    b.push_back((uint8_t)(v >> 16));
    b.push_back((uint8_t)(v >> 8));
    b.push_back((uint8_t)v);
}

void png_chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
    put_be32(out, (uint32_t)data.size());
    std::vector<uint8_t> td(type, type + 4);
    td.insert(td.end(), data.begin(), data.end());
    out.insert(out.end(), td.begin(), td.end());
    put_be32(out, crc32_update(0u, td.data(), td.size()));
}

}  // namespace
}  // namespace oks

extern "C" {

int okscuda_percentile(okscuda_ctx* ctx, const float* d_vals, long long n, float pct, float* h_out) {
    OKS_CHECK_CTX();
    if (!h_out || n < 0 || (n > 0 && !d_vals)) return set_err(ctx, OKS_EINVAL, "percentile: bad arguments");
    *h_out = 0.0f;
    if (n == 0) return OKS_OK;   // main.rs:1148-1150
    // main.rs:1151-1152 in f32: round(pct / 100 * (n - 1)) (half away from zero), clamped to n - 1
    const float fk = std::round((pct / 100.0f) * (float)(n - 1));
    unsigned long long k = fk > 0.0f ? (unsigned long long)fk : 0ull;   // `as usize` saturates at 0
    if (k > (unsigned long long)(n - 1)) k = (unsigned long long)(n - 1);
    oks::SelectState* st = nullptr;
    OKS_CUDA(cudaMallocAsync(&st, sizeof(oks::SelectState), ctx->stream));
    oks::SelectState h{};
    h.rank = k;
    cudaError_t e = cudaMemcpyAsync(st, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream);
    const int threads = 256;
    const long long blocks = std::min<long long>((n + threads - 1) / threads, 148ll * 8);
    for (int shift = 24; shift >= 0 && e == cudaSuccess; shift -= 8) {
        ProfScope ps(ctx, "k_select");
        oks::k_select_hist<<<(unsigned)blocks, threads, 0, ctx->stream>>>(d_vals, n, st, shift);
        oks::k_select_pick<<<1, 1, 0, ctx->stream>>>(st, shift);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(st, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_err(ctx, e, "percentile");
    // the selected key back to its float
    const uint32_t key = h.prefix;
    const uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
    std::memcpy(h_out, &u, sizeof u);
    return OKS_OK;
}

int okscuda_window_u8(okscuda_ctx* ctx, const float* d_img, long long n, float lo, float hi, int gamma,
                      uint8_t* d_out) {
    OKS_CHECK_CTX();
    if (n < 0 || (n > 0 && (!d_img || !d_out))) return set_err(ctx, OKS_EINVAL, "window_u8: bad arguments");
    if (n == 0) return OKS_OK;
    hi = std::max(hi, lo + FLT_EPSILON);   // main.rs:1097, 1125 (f32)
    const int threads = 256;
    const long long blocks = std::min<long long>((n + threads - 1) / threads, 148ll * 16);
    ProfScope ps(ctx, "k_window_u8");
    oks::k_window_u8<<<(unsigned)blocks, threads, 0, ctx->stream>>>(d_img, n, lo, hi, gamma != 0, d_out);
    OKS_CUDA(cudaGetLastError());
    return OKS_OK;
}

int okscuda_write_nifti(const float* h_vol, int nz, int ny, int nx, const char* path) {
    if (!h_vol || !path || nz <= 0 || ny <= 0 || nx <= 0) return OKS_EINVAL;
    if (nz > 32767 || ny > 32767 || nx > 32767) return OKS_ESHAPE;   // dims are i16 (main.rs:1041-1043)
    uint8_t hdr[348] = {};
    auto put16 = [&](int off, int16_t v) { std::memcpy(hdr + off, &v, 2); };
    auto put32 = [&](int off, const void* v) { std::memcpy(hdr + off, v, 4); };
    const int32_t sizeof_hdr = 348;
    put32(0, &sizeof_hdr);
    const int16_t dims[8] = {3, (int16_t)nx, (int16_t)ny, (int16_t)nz, 1, 1, 1, 1};
    for (int i = 0; i < 8; ++i) put16(40 + 2 * i, dims[i]);
    put16(70, 16);                                   // DT_FLOAT32
    put16(72, 32);                                   // bitpix
    const float pixdim[8] = {1.f, 1.f, 1.f, 1.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < 8; ++i) put32(76 + 4 * i, &pixdim[i]);
    const float vox_offset = 352.0f, slope = 1.0f;
    put32(108, &vox_offset);
    put32(112, &slope);
    std::memcpy(hdr + 344, "n+1\0", 4);
    FILE* f = std::fopen(path, "wb");
    if (!f) return OKS_EINVAL;
    const uint8_t ext[4] = {0, 0, 0, 0};
    const size_t nvox = (size_t)nz * ny * nx;
    bool ok = std::fwrite(hdr, 1, 348, f) == 348 && std::fwrite(ext, 1, 4, f) == 4 &&
              std::fwrite(h_vol, sizeof(float), nvox, f) == nvox;   // little-endian host: x fastest
    ok = (std::fclose(f) == 0) && ok;
    return ok ? OKS_OK : OKS_EINVAL;
}

int okscuda_write_png(const uint8_t* h_gray, int width, int height, const char* path) {
    if (!h_gray || !path || width <= 0 || height <= 0) return OKS_EINVAL;
    using oks::put_be32;
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});        // 8-bit, grayscale, deflate, filter 0, no interlace
    oks::png_chunk(png, "IHDR", ihdr);
    // raw scanlines (filter type 0) in a zlib stream of stored deflate blocks
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (width + 1));
    for (int y = 0; y < height; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), h_gray + (size_t)y * width, h_gray + (size_t)(y + 1) * width);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;                           // Adler-32 of the raw bytes
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)(len & 255));
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)(~len & 255));
        z.push_back((uint8_t)((~len >> 8) & 255));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        if (last) break;
    }
    put_be32(z, (b << 16) | a);
    oks::png_chunk(png, "IDAT", z);
    oks::png_chunk(png, "IEND", {});
    FILE* f = std::fopen(path, "wb");
    if (!f) return OKS_EINVAL;
    bool ok = std::fwrite(png.data(), 1, png.size(), f) == png.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? OKS_OK : OKS_EINVAL;
}

}  // extern "C"
