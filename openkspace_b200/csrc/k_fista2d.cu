// sm_100a FISTA for arbitrary 2-D sampling masks (cs.rs:59-139 when the
// mask is not constant along kx -- e.g. the partial rows the reference's
// reader produces after readout-oversampling removal, reader.rs:394-457).
//
// Modulated form (D2 = diag((-1)^{r+x}), s = (-1)^{ny/2 + nx/2}, N = ny nx):
//   F2c = s D2 F2 D2 / sqrt(N)  =>  F2c^H M (F2c z - y) = D2 h,
//   h = F2^H [m' (F2 z~ - y')],  z~ = D2 z,  y' = s sqrt(N) D2 y,  m' = M / N.
// The Haar prox of v = D2 (z~ - h) is the plain Haar of v~ = z~ - h with the
// untouched LL band of v landing on the plain HH band of v~.
//
// Per iteration two passes over L2/HBM-resident state (X~, Z~, S):
//   column pass: S <- F_y^H [ m' (F_y S - y') ]           (S holds F_x z~ on entry)
//   row pass   : h = F_x^H S ; v~ = z~ - h ; prox ; momentum -> X~, Z~ ;
//                S <- F_x z~'
// F2 = F_y F_x commute, so together they apply h = F2^H m'(F2 z~ - y').
#include <cuda_runtime.h>

#include "fft_dev.cuh"
#include "kernels.h"

namespace oks {

__device__ __forceinline__ float ysign(int r, int x) { return ((r + x) & 1) ? -1.f : 1.f; }

// ------------------------------------------------------------ column pass
// mode 0 (init): S <- F_y^H (m' y')        mode 1: S <- F_y^H [m' (F_y S - y')]
__global__ void k2d_col(Fista2dArgs a, FftPlan pl, const float2* __restrict__ gtw,
                        const float2* __restrict__ groots, int roots_total, int tc, int mode) {
    extern __shared__ float2 sm[];
    const int n = a.ny, nx = a.nx;
    float2* A = sm;
    float2* B = A + (size_t)tc * n;
    float2* YT = B + (size_t)tc * n;
    float2* TW = YT + (size_t)tc * n;
    float2* RT = TW + pl.tw_total;
    float* MK = reinterpret_cast<float*>(RT + roots_total);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long p = blockIdx.y;
    const int x0 = blockIdx.x * tc;
    const long long mi = (p + a.mask_offset) % a.mask_mod;
    // a tile of kx columns the mask never samples contributes nothing: the
    // row pass reads those columns of S as zero, so skip the tile entirely
    {
        const uint32_t* cb = a.colbits + mi * a.col_wstride;
        bool any = false;
        for (int c = 0; c < tc && x0 + c < nx; ++c) any |= ((cb[(x0 + c) >> 5] >> ((x0 + c) & 31)) & 1u) != 0;
        if (!any) return;
    }
    const float2* y = a.y + p * a.y_stride;
    const uint8_t* mk = a.mask + mi * a.mask_stride;
    float2* S = a.S + p * a.st_stride;
    for (int q = tid; q < pl.tw_total; q += nthr) TW[q] = gtw[q];
    for (int q = tid; q < roots_total; q += nthr) RT[q] = groots[q];
    for (int q = tid; q < tc * n; q += nthr) {
        const int r = q / tc, c = q - r * tc, x = x0 + c;
        float m = 0.f;
        float2 yv = make_float2(0.f, 0.f), sv = make_float2(0.f, 0.f);
        if (x < nx) {
            const long long off = (long long)r * nx + x;
            m = mk[off] ? a.minv : 0.f;
            if (m != 0.f) yv = y[off] * (a.ysc * ysign(r, x));
            if (mode) sv = S[off];
        }
        MK[q] = m;
        YT[q] = yv;
        A[q] = mode ? sv : (m != 0.f ? yv * m : make_float2(0.f, 0.f));
    }
    __syncthreads();
    float2* res;
    if (mode) {
        float2* F = fft_smem<-1, true>(A, A, B, pl, TW, RT, tc, 1, tc, tid, nthr);
        for (int q = tid; q < tc * n; q += nthr) {
            const float m = MK[q];
            F[q] = (m != 0.f) ? (F[q] - YT[q]) * m : make_float2(0.f, 0.f);
        }
        __syncthreads();
        res = fft_smem<+1, true>(F, A, B, pl, TW, RT, tc, 1, tc, tid, nthr);
    } else {
        res = fft_smem<+1, true>(A, A, B, pl, TW, RT, tc, 1, tc, tid, nthr);
    }
    for (int q = tid; q < tc * n; q += nthr) {
        const int r = q / tc, c = q - r * tc, x = x0 + c;
        if (x < nx) S[(long long)r * nx + x] = res[q];
    }
}

// --------------------------------------------------------------- row pass
// rows come in pairs (Haar); rpc rows per CTA (even).
// mode 0 (init): x~0 = z~0 = F_x^H S ; S <- F_x z~0
// mode 1: h = F_x^H S ; prox/momentum ; S <- F_x z~'
__global__ void k2d_row(Fista2dArgs a, FftPlan pl, const float2* __restrict__ gtw,
                        const float2* __restrict__ groots, int roots_total, int rpc, int mode, int it) {
    extern __shared__ float2 sm[];
    const int n = a.nx, ny = a.ny;
    float2* A = sm;
    float2* B = A + (size_t)rpc * n;
    float2* TW = B + (size_t)rpc * n;
    float2* RT = TW + pl.tw_total;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long p = blockIdx.y;
    const int r0 = blockIdx.x * rpc;
    const int nrow = min(rpc, ny - r0);
    float2* S = a.S + p * a.st_stride + (long long)r0 * n;
    float2* X = a.X + p * a.st_stride + (long long)r0 * n;
    float2* Z = a.Z + p * a.st_stride + (long long)r0 * n;
    for (int q = tid; q < pl.tw_total; q += nthr) TW[q] = gtw[q];
    for (int q = tid; q < roots_total; q += nthr) RT[q] = groots[q];
    const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
    for (int q = tid; q < rpc * n; q += nthr) {
        const int x = q % n;
        const bool on = (q / n < nrow) && ((cb[x >> 5] >> (x & 31)) & 1u);
        A[q] = on ? S[q] : make_float2(0.f, 0.f);   // unsampled kx columns of S are zero
    }
    __syncthreads();
    float2* H = fft_smem<+1, false>(A, A, B, pl, TW, RT, rpc, n, 1, tid, nthr);
    float2* O = (H == A) ? B : A;   // the free buffer receives z~'
    if (mode == 0) {
        for (int q = tid; q < nrow * n; q += nthr) {
            const float2 h = H[q];
            X[q] = h;
            Z[q] = h;
            O[q] = h;
        }
        for (int q = nrow * n + tid; q < rpc * n; q += nthr) O[q] = make_float2(0.f, 0.f);
    } else {
        const float alpha = a.alpha[it];
        const float lam = a.lambda;
        const int hx = n / 2;
        for (int q = tid; q < (rpc / 2) * hx; q += nthr) {
            const int i = q / hx, j = q - i * hx;
            const int e0 = (2 * i) * n + 2 * j, e1 = e0 + n;
            if (2 * i >= nrow) {
                O[e0] = O[e0 + 1] = O[e1] = O[e1 + 1] = make_float2(0.f, 0.f);
                continue;
            }
            const float4 za = *reinterpret_cast<const float4*>(Z + e0);
            const float4 zd = *reinterpret_cast<const float4*>(Z + e1);
            const float2 va = make_float2(za.x, za.y) - H[e0], vb = make_float2(za.z, za.w) - H[e0 + 1];
            const float2 vd = make_float2(zd.x, zd.y) - H[e1], ve = make_float2(zd.z, zd.w) - H[e1 + 1];
            const float2 s0 = va + vb, d0 = va - vb, s1 = vd + ve, d1 = vd - ve;
            float2 pll = (s0 + s1) * 0.5f, phl = (d0 + d1) * 0.5f;
            float2 plh = (s0 - s1) * 0.5f, phh = (d0 - d1) * 0.5f;
            // phh is the LL band of the demodulated image: left untouched
            pll = shrink_exact(pll, lam);
            phl = shrink_exact(phl, lam);
            plh = shrink_exact(plh, lam);
            const float2 t0 = pll + plh, t1 = phl + phh, t2 = pll - plh, t3 = phl - phh;
            const float2 xa = (t0 + t1) * 0.5f, xb = (t0 - t1) * 0.5f;
            const float2 xd = (t2 + t3) * 0.5f, xe = (t2 - t3) * 0.5f;
            const float4 xo0 = *reinterpret_cast<const float4*>(X + e0);
            const float4 xo1 = *reinterpret_cast<const float4*>(X + e1);
            const float2 za2 = xa + (xa - make_float2(xo0.x, xo0.y)) * alpha;
            const float2 zb2 = xb + (xb - make_float2(xo0.z, xo0.w)) * alpha;
            const float2 zd2 = xd + (xd - make_float2(xo1.x, xo1.y)) * alpha;
            const float2 ze2 = xe + (xe - make_float2(xo1.z, xo1.w)) * alpha;
            *reinterpret_cast<float4*>(X + e0) = make_float4(xa.x, xa.y, xb.x, xb.y);
            *reinterpret_cast<float4*>(X + e1) = make_float4(xd.x, xd.y, xe.x, xe.y);
            *reinterpret_cast<float4*>(Z + e0) = make_float4(za2.x, za2.y, zb2.x, zb2.y);
            *reinterpret_cast<float4*>(Z + e1) = make_float4(zd2.x, zd2.y, ze2.x, ze2.y);
            O[e0] = za2; O[e0 + 1] = zb2; O[e1] = zd2; O[e1 + 1] = ze2;
        }
    }
    __syncthreads();
    float2* F = fft_smem<-1, false>(O, O, H, pl, TW, RT, rpc, n, 1, tid, nthr);
    for (int q = tid; q < nrow * n; q += nthr) {
        const int x = q % n;
        if ((cb[x >> 5] >> (x & 31)) & 1u) S[q] = F[q];   // only sampled columns are read back
    }
}

// ------------------------------------------------ prox between row DFTs
// The element-wise middle of the row pass when the two row transforms run
// on the tensor cores (k_dft_tc.cu): W = F_x^H S is in global memory.  One
// thread per 2x2 block, the same arithmetic as k2d_row above.
__global__ void k2d_prox(Fista2dArgs a, const float2* __restrict__ W, int mode, int it) {
    const int ny = a.ny, nx = a.nx, hx = nx / 2, hy = ny / 2;
    const long long per = (long long)hy * hx;
    const long long tot = a.nprob * per;
    const float alpha = mode ? __ldg(a.alpha + it) : 0.f;
    const float lam = a.lambda;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
         q += (long long)gridDim.x * blockDim.x) {
        const long long p = q / per, b = q - p * per;
        const int i = (int)(b / hx), j = (int)(b - (long long)i * hx);
        const long long e0 = p * a.st_stride + (long long)(2 * i) * nx + 2 * j, e1 = e0 + nx;
        const float4 h0 = *reinterpret_cast<const float4*>(W + e0);
        const float4 h1 = *reinterpret_cast<const float4*>(W + e1);
        if (mode == 0) {
            *reinterpret_cast<float4*>(a.X + e0) = h0;
            *reinterpret_cast<float4*>(a.X + e1) = h1;
            *reinterpret_cast<float4*>(a.Z + e0) = h0;
            *reinterpret_cast<float4*>(a.Z + e1) = h1;
            continue;
        }
        const float4 za = *reinterpret_cast<const float4*>(a.Z + e0);
        const float4 zd = *reinterpret_cast<const float4*>(a.Z + e1);
        const float4 xo0 = *reinterpret_cast<const float4*>(a.X + e0);
        const float4 xo1 = *reinterpret_cast<const float4*>(a.X + e1);
        const float2 va = make_float2(za.x - h0.x, za.y - h0.y), vb = make_float2(za.z - h0.z, za.w - h0.w);
        const float2 vd = make_float2(zd.x - h1.x, zd.y - h1.y), ve = make_float2(zd.z - h1.z, zd.w - h1.w);
        const float2 s0 = va + vb, d0 = va - vb, s1 = vd + ve, d1 = vd - ve;
        float2 pll = (s0 + s1) * 0.5f, phl = (d0 + d1) * 0.5f;
        float2 plh = (s0 - s1) * 0.5f, phh = (d0 - d1) * 0.5f;
        // phh is the LL band of the demodulated image: left untouched
        pll = shrink_exact(pll, lam);
        phl = shrink_exact(phl, lam);
        plh = shrink_exact(plh, lam);
        const float2 t0 = pll + plh, t1 = phl + phh, t2 = pll - plh, t3 = phl - phh;
        const float2 xa = (t0 + t1) * 0.5f, xb = (t0 - t1) * 0.5f;
        const float2 xd = (t2 + t3) * 0.5f, xe = (t2 - t3) * 0.5f;
        const float2 za2 = xa + (xa - make_float2(xo0.x, xo0.y)) * alpha;
        const float2 zb2 = xb + (xb - make_float2(xo0.z, xo0.w)) * alpha;
        const float2 zd2 = xd + (xd - make_float2(xo1.x, xo1.y)) * alpha;
        const float2 ze2 = xe + (xe - make_float2(xo1.z, xo1.w)) * alpha;
        *reinterpret_cast<float4*>(a.X + e0) = make_float4(xa.x, xa.y, xb.x, xb.y);
        *reinterpret_cast<float4*>(a.X + e1) = make_float4(xd.x, xd.y, xe.x, xe.y);
        *reinterpret_cast<float4*>(a.Z + e0) = make_float4(za2.x, za2.y, zb2.x, zb2.y);
        *reinterpret_cast<float4*>(a.Z + e1) = make_float4(zd2.x, zd2.y, ze2.x, ze2.y);
    }
}

cudaError_t launch_fista2d_prox(const Fista2dArgs& a, const float2* W, int mode, int it, cudaStream_t st) {
    const long long tot = a.nprob * (long long)(a.ny / 2) * (a.nx / 2);
    if (tot <= 0) return cudaSuccess;
    long long blocks = (tot + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k2d_prox<<<(unsigned)blocks, 256, 0, st>>>(a, W, mode, it);
    return cudaGetLastError();
}

// ------------------------------------------------------- demodulated copy
__global__ void k2d_demod(const float2* __restrict__ X, float2* __restrict__ out, long long nprob, int ny, int nx,
                          long long in_stride, long long out_stride) {
    const long long per = (long long)ny * nx;
    const long long tot = nprob * per;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
         q += (long long)gridDim.x * blockDim.x) {
        const long long p = q / per, e = q - p * per;
        const int r = (int)(e / nx), x = (int)(e - (long long)r * nx);
        const float2 v = X[p * in_stride + e];
        out[p * out_stride + e] = ((r + x) & 1) ? make_float2(-v.x, -v.y) : v;
    }
}

static int rup(int v, int m) { return (v + m - 1) / m * m; }

cudaError_t launch_fista2d_col(const Fista2dArgs& a, const DevPlan& py, int mode, cudaStream_t st) {
    const int n = a.ny;
    int tc = 8;
    if ((size_t)3 * tc * n * sizeof(float2) > 150 * 1024) tc = 4;
    if ((size_t)3 * tc * n * sizeof(float2) > 150 * 1024) tc = 1;
    size_t smem = sizeof(float2) * ((size_t)3 * tc * n + py.plan.tw_total + py.roots_total) +
                  sizeof(float) * (size_t)tc * n;
    cudaError_t e = set_smem_attr(reinterpret_cast<const void*>(k2d_col), smem);
    if (e != cudaSuccess) return e;
    int nthr = rup(tc * n / 4, 32);
    nthr = nthr < 64 ? 64 : (nthr > 256 ? 256 : nthr);
    dim3 grid((a.nx + tc - 1) / tc, (unsigned)a.nprob);
    k2d_col<<<grid, nthr, smem, st>>>(a, py.plan, py.tw, py.roots, py.roots_total, tc, mode);
    return cudaGetLastError();
}

cudaError_t launch_fista2d_row(const Fista2dArgs& a, const DevPlan& px, int mode, int it, cudaStream_t st) {
    const int n = a.nx;
    int rpc = 4;
    if ((size_t)2 * rpc * n * sizeof(float2) > 150 * 1024) rpc = 2;
    size_t smem = sizeof(float2) * ((size_t)2 * rpc * n + px.plan.tw_total + px.roots_total);
    cudaError_t e = set_smem_attr(reinterpret_cast<const void*>(k2d_row), smem);
    if (e != cudaSuccess) return e;
    int nthr = rup(rpc * n / 4, 32);
    nthr = nthr < 64 ? 64 : (nthr > 256 ? 256 : nthr);
    dim3 grid((a.ny + rpc - 1) / rpc, (unsigned)a.nprob);
    k2d_row<<<grid, nthr, smem, st>>>(a, px.plan, px.tw, px.roots, px.roots_total, rpc, mode, it);
    return cudaGetLastError();
}

cudaError_t launch_fista2d_demod(const float2* X, float2* out, long long nprob, int ny, int nx, long long in_stride,
                                 long long out_stride, cudaStream_t st) {
    const long long tot = nprob * ny * nx;
    if (tot <= 0) return cudaSuccess;
    long long blocks = (tot + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k2d_demod<<<(unsigned)blocks, 256, 0, st>>>(X, out, nprob, ny, nx, in_stride, out_stride);
    return cudaGetLastError();
}

}  // namespace oks
