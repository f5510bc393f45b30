// Image-domain SENSE unfolding and g-factor for regular 1-D undersampling
// along ky (openkspace-recon/src/sense.rs:64-252) on the device.
//
// One thread per reduced voxel (y0, x), y0 < ny / R, x fastest (coalesced map
// and image reads).  Per voxel, in f32 and in the reference's operation order:
//   C[c][k] = S_c(y0 + k ny/R, x)                      (sense.rs:107-111)
//   A = C^H C + ridge I, lower triangle                (sense.rs:114-126)
//   b = R C^H a,  a[c] = I_c(y0, x)                     (sense.rs:129-136)
//   L = chol(A), L^-1 by forward substitution, rho = L^-H (L^-1 b)
//                      (prewhiten.rs:148-210, sense.rs:141-166)
//   out(y0 + k ny/R, x) = rho[k];  g = sqrt(max(diag((C^H C)^-1) A_kk, 0))
//                      (sense.rs:170-175, 236-247)
// A voxel whose Cholesky or triangular inverse fails stays zero, as in the
// reference.  Every product and sum is an explicitly rounded intrinsic
// (__fmul_rn, __fadd_rn, ...), never contracted into a fused multiply-add,
// and division and square root are IEEE-rounded, so the device computes the
// same f32 values as a sequential f32 implementation of the same order.
#include <cfloat>

#include "ctx.h"

namespace oks {
namespace {

struct C32 {
    float re, im;
};
__device__ __forceinline__ C32 cadd(C32 a, C32 b) { return {__fadd_rn(a.re, b.re), __fadd_rn(a.im, b.im)}; }
__device__ __forceinline__ C32 csub(C32 a, C32 b) { return {__fsub_rn(a.re, b.re), __fsub_rn(a.im, b.im)}; }
// num_complex multiplication: (a.re b.re - a.im b.im, a.re b.im + a.im b.re)
__device__ __forceinline__ C32 cmul(C32 a, C32 b) {
    return {__fsub_rn(__fmul_rn(a.re, b.re), __fmul_rn(a.im, b.im)),
            __fadd_rn(__fmul_rn(a.re, b.im), __fmul_rn(a.im, b.re))};
}
__device__ __forceinline__ C32 conj(C32 a) { return {a.re, -a.im}; }
// num_complex division: ((a.re b.re + a.im b.im) / |b|^2, (a.im b.re - a.re b.im) / |b|^2)
__device__ __forceinline__ C32 cdiv(C32 a, C32 b) {
    const float n = __fadd_rn(__fmul_rn(b.re, b.re), __fmul_rn(b.im, b.im));
    return {__fdiv_rn(__fadd_rn(__fmul_rn(a.re, b.re), __fmul_rn(a.im, b.im)), n),
            __fdiv_rn(__fsub_rn(__fmul_rn(a.im, b.re), __fmul_rn(a.re, b.im)), n)};
}
__device__ __forceinline__ C32 ld(const float2* p) {
    const float2 v = __ldg(p);
    return {v.x, v.y};
}

// Lower-triangular index of (i, j), j <= i.
__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

template <int R>
__global__ void k_sense_unfold(const float2* __restrict__ aliased, const float2* __restrict__ maps, int nc, int ny,
                               int nx, float ridge, float2* __restrict__ out, float* __restrict__ gout) {
    const int ny_red = ny / R;
    const long long npix = (long long)ny_red * nx;
    const long long plane = (long long)ny * nx;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npix;
         q += (long long)gridDim.x * blockDim.x) {
        const int y0 = (int)(q / nx), x = (int)(q - (long long)y0 * nx);
        C32 A[tri(R, 0)];                     // C^H C + ridge I, lower triangle; then L in place
        for (int a = 0; a < R; ++a)
            for (int b = 0; b <= a; ++b) {
                C32 acc = {0.f, 0.f};
                for (int c = 0; c < nc; ++c) {
                    const C32 ca = ld(maps + c * plane + (long long)(y0 + a * ny_red) * nx + x);
                    const C32 cb = ld(maps + c * plane + (long long)(y0 + b * ny_red) * nx + x);
                    acc = cadd(acc, cmul(conj(ca), cb));
                }
                if (a == b) acc = cadd(acc, C32{ridge, 0.f});
                A[tri(a, b)] = acc;
            }
        float adiag[R];
#pragma unroll
        for (int k = 0; k < R; ++k) adiag[k] = A[tri(k, k)].re;
        C32 rhs[R];
        if (out) {
            for (int a = 0; a < R; ++a) {
                C32 acc = {0.f, 0.f};
                for (int c = 0; c < nc; ++c) {
                    const C32 ca = ld(maps + c * plane + (long long)(y0 + a * ny_red) * nx + x);
                    acc = cadd(acc, cmul(conj(ca), ld(aliased + c * plane + (long long)y0 * nx + x)));
                }
                rhs[a] = cmul(acc, C32{(float)R, 0.f});
            }
        }
        // Cholesky, prewhiten.rs:148-179 (column i of L overwrites column i of A)
        bool ok = true;
        for (int i = 0; i < R && ok; ++i) {
            C32 diag = A[tri(i, i)];
            for (int k = 0; k < i; ++k) diag = csub(diag, cmul(A[tri(i, k)], conj(A[tri(i, k)])));
            const float d_re = diag.re;
            if (!isfinite(d_re) || d_re <= 0.f) {
                ok = false;
                break;
            }
            const float l_ii = __fsqrt_rn(d_re);
            A[tri(i, i)] = C32{l_ii, 0.f};
            const C32 inv_l_ii = {__fdiv_rn(1.f, l_ii), 0.f};
            for (int j = i + 1; j < R; ++j) {
                C32 s = A[tri(j, i)];
                for (int k = 0; k < i; ++k) s = csub(s, cmul(A[tri(j, k)], conj(A[tri(i, k)])));
                A[tri(j, i)] = cmul(s, inv_l_ii);
            }
        }
        if (!ok) continue;                    // the voxel stays zero (sense.rs:141-143)
        // L^-1 by forward substitution on each unit column, prewhiten.rs:183-210
        // (the whole column is solved, entries above the diagonal included, as
        // the reference does before it clears the strict upper triangle)
        C32 V[tri(R, 0)];
        for (int col = 0; col < R && ok; ++col) {
            C32 xc[R];
            for (int i = 0; i < R; ++i) {
                C32 s = {i == col ? 1.f : 0.f, 0.f};
                for (int j = 0; j < i; ++j) s = csub(s, cmul(A[tri(i, j)], xc[j]));
                const C32 d = A[tri(i, i)];
                if (fabsf(d.re) < FLT_EPSILON && fabsf(d.im) < FLT_EPSILON) {
                    ok = false;
                    break;
                }
                xc[i] = cdiv(s, d);
                if (i >= col) V[tri(i, col)] = xc[i];
            }
        }
        if (!ok) continue;
        if (out) {
            C32 tmp[R];
            for (int i = 0; i < R; ++i) {     // tmp = L^-1 rhs
                C32 acc = {0.f, 0.f};
                for (int j = 0; j <= i; ++j) acc = cadd(acc, cmul(V[tri(i, j)], rhs[j]));
                tmp[i] = acc;
            }
            for (int i = 0; i < R; ++i) {     // rho = L^-H tmp, scattered to the aliased rows
                C32 acc = {0.f, 0.f};
                for (int j = i; j < R; ++j) acc = cadd(acc, cmul(conj(V[tri(j, i)]), tmp[j]));
                out[(long long)(y0 + i * ny_red) * nx + x] = make_float2(acc.re, acc.im);
            }
        }
        if (gout) {
            for (int k = 0; k < R; ++k) {     // sense.rs:236-247
                float inv_diag = 0.f;
                for (int j = k; j < R; ++j) {
                    const C32 v = V[tri(j, k)];
                    inv_diag = __fadd_rn(inv_diag, __fadd_rn(__fmul_rn(v.re, v.re), __fmul_rn(v.im, v.im)));
                }
                const float chc_diag = fmaxf(adiag[k], 0.f);
                gout[(long long)(y0 + k * ny_red) * nx + x] = __fsqrt_rn(fmaxf(__fmul_rn(inv_diag, chc_diag), 0.f));
            }
        }
    }
}

template <int R>
cudaError_t launch_unfold(const float2* al, const float2* maps, int nc, int ny, int nx, float ridge, float2* out,
                          float* g, cudaStream_t st) {
    const long long npix = (long long)(ny / R) * nx;
    const int threads = 128;
    const long long blocks = std::min<long long>((npix + threads - 1) / threads, 148ll * 32);
    if (blocks < 1) return cudaSuccess;
    k_sense_unfold<R><<<(unsigned)blocks, threads, 0, st>>>(al, maps, nc, ny, nx, ridge, out, g);
    return cudaGetLastError();
}

}  // namespace
}  // namespace oks

extern "C" int okscuda_sense_unfold(okscuda_ctx* ctx, const okscuda_c64* d_aliased, const okscuda_c64* d_maps, int nc,
                                    int ny, int nx, int r, float ridge, okscuda_c64* d_out, float* d_gfactor) {
    OKS_CHECK_CTX();
    if (r < 1) return set_err(ctx, OKS_EINVAL, "SENSE: acceleration factor must be >= 1");
    if (nc < 0 || ny < 0 || nx < 0 || !d_maps || (!d_out && !d_gfactor) || (d_out && !d_aliased))
        return set_err(ctx, OKS_EINVAL, "sense_unfold: bad arguments");
    if (ny % r != 0) return set_err(ctx, OKS_ESHAPE, "SENSE: Ny (%d) must be divisible by R (%d)", ny, r);
    if (r > 8) return set_err(ctx, OKS_ENOTSUP, "sense_unfold: R <= 8 (R = %d)", r);
    const size_t npix = (size_t)ny * nx;
    if (d_out) OKS_CUDA(cudaMemsetAsync(d_out, 0, sizeof(okscuda_c64) * npix, ctx->stream));
    if (d_gfactor) OKS_CUDA(cudaMemsetAsync(d_gfactor, 0, sizeof(float) * npix, ctx->stream));
    if (nc == 0 || nx == 0 || ny == 0) return OKS_OK;
    const float2* al = reinterpret_cast<const float2*>(d_aliased);
    const float2* mp = reinterpret_cast<const float2*>(d_maps);
    float2* o = reinterpret_cast<float2*>(d_out);
    cudaError_t e;
    ProfScope ps(ctx, "k_sense_unfold");
    switch (r) {
        case 1: e = oks::launch_unfold<1>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 2: e = oks::launch_unfold<2>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 3: e = oks::launch_unfold<3>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 4: e = oks::launch_unfold<4>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 5: e = oks::launch_unfold<5>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 6: e = oks::launch_unfold<6>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        case 7: e = oks::launch_unfold<7>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
        default: e = oks::launch_unfold<8>(al, mp, nc, ny, nx, ridge, o, d_gfactor, ctx->stream); break;
    }
    if (e != cudaSuccess) return cuda_err(ctx, e, "sense_unfold");
    return OKS_OK;
}
