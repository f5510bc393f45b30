// sm_100a kernels of the FISTA-CS path (generic, shared-memory resident).
//
// Reference routines (crates/openkspace-recon/src/):
//   cs.rs:59-139     fista_cs_single_coil    -> k_fista_col
//   cs.rs:141-218    centred_fft2/ifft2      -> k_row_xform + k_col_xform
//   wavelet.rs:32-99 Haar + soft-threshold   -> fused in k_fista_col; k_haar, k_soft_threshold
//   strategy.rs:870-885 RSS + crop           -> k_rss
//
// Separable form used by k_fista_col.  For a ky-only mask M = diag(m) (x) I
// the 2-D gradient F^H M (F z - y) equals, column by column,
// F_y^H m (F_y z - yhat) with yhat = F_x^H y (a row IDFT done once).  With
// the centred unitary DFT written F_c = (-1)^{n/2} D F D / sqrt(n),
// D = diag((-1)^r), the iteration runs on modulated state z~ = D z with plain
// DFTs: h = F^H [m' (F z~ - y')], m' = m / n, y' = sqrt(n) (-1)^{n/2} D yhat,
// v~ = z~ - h.  The Haar prox of v = D v~ equals the plain Haar of v~ with the
// roles of the bands permuted: the untouched LL band of v is the
// "row-difference, column-sum" band of v~.  Momentum is linear, so the state
// stays modulated; the output is x = D x~.
#include <cuda_runtime.h>

#include "fft_dev.cuh"
#include "kernels.h"

namespace oks {

// ------------------------------------------------------------------ rows
__global__ void k_row_xform(RowXformArgs a, FftPlan pl, const float2* __restrict__ gtw,
                            const float2* __restrict__ groots, int roots_total, int rpc) {
    extern __shared__ float2 sm[];
    const int n = pl.n;
    float2* A = sm;
    float2* B = A + (size_t)rpc * n;
    float2* TW = B + (size_t)rpc * n;
    float2* RT = TW + pl.tw_total;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int q = tid; q < pl.tw_total; q += nthr) TW[q] = gtw[q];
    for (int q = tid; q < roots_total; q += nthr) RT[q] = groots[q];
    const long long row0 = (long long)blockIdx.x * rpc;
    const int c1 = a.centred ? (n + 1) / 2 : 0;   // ifftshift: rotate left by ceil(n/2)
    const int c2 = a.centred ? n / 2 : 0;         // fftshift:  rotate left by floor(n/2)
    for (int q = tid; q < rpc * n; q += nthr) {
        const int lr = q / n, m = q - lr * n;
        const long long row = row0 + lr;
        float2 v = make_float2(0.f, 0.f);
        if (row < a.nrows) {
            if (!a.use_keep || row_on(a.keep, row / a.rows_per_prob, (int)(row % a.rows_per_prob))) {
                int src = m + c1;
                if (src >= n) src -= n;
                v = a.in[row * a.ld_in + src];
            }
        }
        A[q] = v;
    }
    __syncthreads();
    float2* res = (a.sign < 0) ? fft_smem<-1, false>(A, A, B, pl, TW, RT, rpc, n, 1, tid, nthr)
                               : fft_smem<+1, false>(A, A, B, pl, TW, RT, rpc, n, 1, tid, nthr);
    for (int q = tid; q < rpc * n; q += nthr) {
        const int lr = q / n, k = q - lr * n;
        const long long row = row0 + lr;
        if (row >= a.nrows) continue;
        int src = k + c2;
        if (src >= n) src -= n;
        float s = a.scale;
        if (a.rowsign && ((row % a.rows_per_prob) & 1)) s = -s;
        a.out[row * a.ld_out + k] = res[lr * n + src] * s;
    }
}

static int round_up(int v, int m) { return (v + m - 1) / m * m; }

cudaError_t launch_row_xform(const RowXformArgs& a, const DevPlan& pl, cudaStream_t st) {
    const int n = pl.plan.n;
    if (a.nrows <= 0) return cudaSuccess;
    if (a.reg && xform_reg_supported(n)) return launch_row_xform_reg(a, n, st);
    int rpc = 16384 / (2 * n);       // two ping-pong buffers within ~128 KB
    if (rpc < 1) rpc = 1;
    if (rpc > 32) rpc = 32;
    if (rpc > a.nrows) rpc = (int)a.nrows;
    size_t smem = sizeof(float2) * ((size_t)2 * rpc * n + pl.plan.tw_total + pl.roots_total);
    cudaError_t e = cudaFuncSetAttribute(k_row_xform, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int nthr = round_up(rpc * n / 2, 32);
    if (nthr > 256) nthr = 256;
    if (nthr < 32) nthr = 32;
    long long grid = (a.nrows + rpc - 1) / rpc;
    k_row_xform<<<(unsigned)grid, nthr, smem, st>>>(a, pl.plan, pl.tw, pl.roots, pl.roots_total, rpc);
    return cudaGetLastError();
}

// --------------------------------------------------------------- columns
__global__ void k_col_xform(ColXformArgs a, FftPlan pl, const float2* __restrict__ gtw,
                            const float2* __restrict__ groots, int roots_total, int tc) {
    extern __shared__ float2 sm[];
    const int n = pl.n;
    float2* A = sm;
    float2* B = A + (size_t)tc * n;
    float2* TW = B + (size_t)tc * n;
    float2* RT = TW + pl.tw_total;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int q = tid; q < pl.tw_total; q += nthr) TW[q] = gtw[q];
    for (int q = tid; q < roots_total; q += nthr) RT[q] = groots[q];
    const int x0 = blockIdx.x * tc;
    float2* base = a.data + (long long)blockIdx.y * a.prob_stride;
    const int c1 = a.centred ? (n + 1) / 2 : 0, c2 = a.centred ? n / 2 : 0;
    for (int q = tid; q < tc * n; q += nthr) {
        const int r = q / tc, c = q - r * tc;
        int src = r + c1;
        if (src >= n) src -= n;
        A[q] = (x0 + c < a.nx) ? base[(long long)src * a.nx + x0 + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* res = (a.sign < 0) ? fft_smem<-1, true>(A, A, B, pl, TW, RT, tc, 1, tc, tid, nthr)
                               : fft_smem<+1, true>(A, A, B, pl, TW, RT, tc, 1, tc, tid, nthr);
    for (int q = tid; q < tc * n; q += nthr) {
        const int k = q / tc, c = q - k * tc;
        if (x0 + c >= a.nx) continue;
        int src = k + c2;
        if (src >= n) src -= n;
        base[(long long)k * a.nx + x0 + c] = res[src * tc + c] * a.scale;
    }
}

cudaError_t launch_col_xform(const ColXformArgs& a, const DevPlan& pl, cudaStream_t st) {
    const int n = pl.plan.n;
    if (a.nprob <= 0 || a.nx <= 0) return cudaSuccess;
    // the register kernel moves 16-byte chunks of two columns
    if (a.reg && xform_reg_supported(n) && (a.nx & 1) == 0 && (a.prob_stride & 1) == 0 &&
        (reinterpret_cast<uintptr_t>(a.data) & 15) == 0)
        return launch_col_xform_reg(a, st);
    int tc = 4096 / n;
    if (tc > 16) tc = 16;
    if (tc < 1) tc = 1;
    size_t smem = sizeof(float2) * ((size_t)2 * tc * n + pl.plan.tw_total + pl.roots_total);
    cudaError_t e = cudaFuncSetAttribute(k_col_xform, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nx + tc - 1) / tc, (unsigned)a.nprob);
    k_col_xform<<<grid, 256, smem, st>>>(a, pl.plan, pl.tw, pl.roots, pl.roots_total, tc);
    return cudaGetLastError();
}

// ----------------------------------------------------- fused column FISTA

__global__ void k_fista_col(FistaColArgs a, FftPlan pl, const float2* __restrict__ gtw,
                            const float2* __restrict__ groots, int roots_total) {
    extern __shared__ float2 sm[];
    const int n = a.ny, n2 = 2 * n, nx = a.nx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    float2* W0 = sm;
    float2* W1 = W0 + n2;
    float2* X = W1 + n2;
    float2* Z = X + n2;
    float2* Y = Z + n2;
    float2* TW = Y + n2;
    float2* RT = TW + pl.tw_total;
    float* M = reinterpret_cast<float*>(RT + roots_total);

    const int j = blockIdx.x;
    const long long b = blockIdx.y;
    const float2* yin = a.ytil + b * a.prob_stride + 2 * j;
    for (int q = tid; q < pl.tw_total; q += nthr) TW[q] = gtw[q];
    for (int q = tid; q < roots_total; q += nthr) RT[q] = groots[q];
    for (int r = tid; r < n; r += nthr) M[r] = row_on(a.mask, b, r) ? a.minv : 0.f;
    for (int q = tid; q < n2; q += nthr) Y[q] = yin[(long long)(q >> 1) * nx + (q & 1)];
    __syncthreads();

    // x~0 = z~0 = F^H (m' y')          (cs.rs:84-96 in modulated form)
    for (int q = tid; q < n2; q += nthr) {
        const float m = M[q >> 1];
        W0[q] = (m != 0.f) ? Y[q] * m : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* H = fft_smem<+1, true>(W0, W0, W1, pl, TW, RT, 2, 1, 2, tid, nthr);
    for (int q = tid; q < n2; q += nthr) { X[q] = H[q]; Z[q] = H[q]; }
    __syncthreads();

    const float lam = a.lambda;
    for (int it = 0; it < a.iters; ++it) {
        // gradient: h = F^H [m' (F z~ - y')]           (cs.rs:101-112)
        float2* F = fft_smem<-1, true>(Z, W0, W1, pl, TW, RT, 2, 1, 2, tid, nthr);
        for (int q = tid; q < n2; q += nthr) {
            const float m = M[q >> 1];
            F[q] = (m != 0.f) ? (F[q] - Y[q]) * m : make_float2(0.f, 0.f);
        }
        __syncthreads();
        H = fft_smem<+1, true>(F, W0, W1, pl, TW, RT, 2, 1, 2, tid, nthr);
        const float alpha = a.alpha[it];
        // prox + momentum on 2x2 blocks (cs.rs:114-136, wavelet.rs:32-99)
        for (int i = tid; i < n / 2; i += nthr) {
            const int q = 4 * i;   // (row 2i, col 0), (2i, 1), (2i+1, 0), (2i+1, 1)
            const float2 va = Z[q] - H[q], vb = Z[q + 1] - H[q + 1];
            const float2 vd = Z[q + 2] - H[q + 2], ve = Z[q + 3] - H[q + 3];
            const float2 s0 = va + vb, d0 = va - vb, s1 = vd + ve, d1 = vd - ve;
            float2 pll = (s0 + s1) * 0.5f, phl = (d0 + d1) * 0.5f;
            float2 plh = (s0 - s1) * 0.5f, phh = (d0 - d1) * 0.5f;
            // plh is the LL band of the demodulated image: left untouched
            pll = shrink_exact(pll, lam);
            phl = shrink_exact(phl, lam);
            phh = shrink_exact(phh, lam);
            const float2 t0 = pll + plh, t1 = phl + phh, t2 = pll - plh, t3 = phl - phh;
            const float2 xa = (t0 + t1) * 0.5f, xb = (t0 - t1) * 0.5f;
            const float2 xd = (t2 + t3) * 0.5f, xe = (t2 - t3) * 0.5f;
            const float2 oa = X[q], ob = X[q + 1], od = X[q + 2], oe = X[q + 3];
            Z[q] = xa + (xa - oa) * alpha;
            Z[q + 1] = xb + (xb - ob) * alpha;
            Z[q + 2] = xd + (xd - od) * alpha;
            Z[q + 3] = xe + (xe - oe) * alpha;
            X[q] = xa; X[q + 1] = xb; X[q + 2] = xd; X[q + 3] = xe;
        }
        __syncthreads();
    }
    float2* xo = a.xout + b * a.out_stride + 2 * j;
    for (int q = tid; q < n2; q += nthr) {
        const int r = q >> 1;
        float2 v = X[q];
        if (r & 1) v = make_float2(-v.x, -v.y);
        xo[(long long)r * nx + (q & 1)] = v;
    }
}

cudaError_t launch_fista_col(const FistaColArgs& a, const DevPlan& pl, cudaStream_t st) {
    if (a.nprob <= 0 || a.nx <= 0) return cudaSuccess;
    const int n = a.ny;
    size_t smem = sizeof(float2) * ((size_t)10 * n + pl.plan.tw_total + pl.roots_total) +
                  sizeof(float) * (size_t)n;
    cudaError_t e = cudaFuncSetAttribute(k_fista_col, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int nthr = round_up(n / 2, 32);
    if (nthr < 64) nthr = 64;
    if (nthr > 256) nthr = 256;
    dim3 grid(a.nx / 2, (unsigned)a.nprob);
    k_fista_col<<<grid, nthr, smem, st>>>(a, pl.plan, pl.tw, pl.roots, pl.roots_total);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ RSS
__global__ void k_rss(RssArgs a) {
    const long long per = (long long)a.ty * a.tx;
    const long long npix = per * a.nslice;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npix;
         q += (long long)gridDim.x * blockDim.x) {
        const long long sl = q / per;
        const long long rem = q - sl * per;
        const int y = (int)(rem / a.tx), x = (int)(rem - (long long)y * a.tx);
        const long long src = sl * a.slice_stride + (long long)(a.y0 + y) * a.nx + (a.x0 + x);
        float s = 0.f;
        for (int c = 0; c < a.nc; ++c) {
            const float2 v = a.coils[c * a.coil_stride + src];
            s += v.x * v.x + v.y * v.y;    // norm_sqr, coil order (strategy.rs:873-876)
        }
        a.out[q] = sqrtf(s);
    }
}

cudaError_t launch_rss(const RssArgs& a, cudaStream_t st) {
    const long long npix = (long long)a.ty * a.tx * a.nslice;
    if (npix <= 0) return cudaSuccess;
    long long blocks = (npix + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_rss<<<(unsigned)blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// ----------------------------------------------------------- Haar prims
__global__ void k_haar(const float2* __restrict__ in, float2* __restrict__ out, long long nprob, int ny,
                       int nx, int inverse) {
    const int hy = ny / 2, hx = nx / 2;
    const long long nblk = nprob * hy * hx;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nblk;
         q += (long long)gridDim.x * blockDim.x) {
        const long long b = q / ((long long)hy * hx);
        const int rem = (int)(q - b * hy * hx);
        const int i = rem / hx, j = rem - i * hx;
        const float2* s = in + b * ny * nx;
        float2* d = out + b * ny * nx;
        if (!inverse) {   // wavelet.rs:39-49
            const float2 pa = s[(2 * i) * nx + 2 * j], pb = s[(2 * i) * nx + 2 * j + 1];
            const float2 pd = s[(2 * i + 1) * nx + 2 * j], pe = s[(2 * i + 1) * nx + 2 * j + 1];
            d[i * nx + j] = (pa + pb + pd + pe) * 0.5f;
            d[i * nx + hx + j] = (pa - pb + pd - pe) * 0.5f;
            d[(hy + i) * nx + j] = (pa + pb - pd - pe) * 0.5f;
            d[(hy + i) * nx + hx + j] = (pa - pb - pd + pe) * 0.5f;
        } else {          // wavelet.rs:62-72
            const float2 ll = s[i * nx + j], hl = s[i * nx + hx + j];
            const float2 lh = s[(hy + i) * nx + j], hh = s[(hy + i) * nx + hx + j];
            d[(2 * i) * nx + 2 * j] = (ll + hl + lh + hh) * 0.5f;
            d[(2 * i) * nx + 2 * j + 1] = (ll - hl + lh - hh) * 0.5f;
            d[(2 * i + 1) * nx + 2 * j] = (ll + hl - lh - hh) * 0.5f;
            d[(2 * i + 1) * nx + 2 * j + 1] = (ll - hl - lh + hh) * 0.5f;
        }
    }
}

cudaError_t launch_haar(const float2* in, float2* out, long long nprob, int ny, int nx, int inverse,
                        cudaStream_t st) {
    const long long nblk = nprob * (ny / 2) * (nx / 2);
    if (nblk <= 0) return cudaSuccess;
    long long blocks = (nblk + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_haar<<<(unsigned)blocks, 256, 0, st>>>(in, out, nprob, ny, nx, inverse);
    return cudaGetLastError();
}

__global__ void k_soft_threshold(float2* d, long long nprob, int ny, int nx, float lam) {
    const long long tot = nprob * ny * nx;
    const int hy = ny / 2, hx = nx / 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
         q += (long long)gridDim.x * blockDim.x) {
        const long long rem = q % ((long long)ny * nx);
        const int i = (int)(rem / nx), j = (int)(rem - (long long)i * nx);
        if (i < hy && j < hx) continue;   // keep LL (wavelet.rs:86-88)
        d[q] = shrink_exact(d[q], lam);
    }
}

cudaError_t launch_soft_threshold(float2* data, long long nprob, int ny, int nx, float lambda,
                                  cudaStream_t st) {
    const long long tot = nprob * ny * nx;
    if (tot <= 0) return cudaSuccess;
    long long blocks = (tot + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_soft_threshold<<<(unsigned)blocks, 256, 0, st>>>(data, nprob, ny, nx, lambda);
    return cudaGetLastError();
}

}  // namespace oks
