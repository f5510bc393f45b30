// SENSE extension mode (north of the reference's per-coil cs; cs.rs:23-26
// names it as the follow-up): coil maps by Walsh's method and the Lipschitz
// constant of the SENSE operator by an FP64 power iteration.
//   sensitivity.rs:37-142  walsh_sensitivity_maps  -> k_walsh (warp per pixel,
//                          lane = coil, f32 like the reference), plus
//                          normalisation to unit root-sum-of-squares
//   (new)                  ||A||^2, A = M F S   -> k_sense_normal_fp64 + norms
#include <cuda_runtime.h>

#include "kernels.h"

namespace oks {

__device__ __forceinline__ float2 cm(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cmc(float2 a, float2 b) {   // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 shfl2(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ float wsum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// imgs, maps: [nc][ny][nx]; one warp per pixel, lane c holds coil c (nc <= 32).
__global__ void k_walsh(const float2* __restrict__ imgs, float2* __restrict__ maps, int nc, int ny, int nx, int window,
                        int power_iters, int normalise) {
    const long long npix = (long long)ny * nx;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int c = threadIdx.x & 31;
    if (warp >= npix) return;                      // whole warp
    const int y = (int)(warp / nx), x = (int)(warp - (long long)y * nx);
    const bool on = c < nc;
    const int y0 = max(y - window, 0), y1 = min(y + window + 1, ny);
    const int x0 = max(x - window, 0), x1 = min(x + window + 1, nx);
    // row c of R = sum over the window of s s^H   (sensitivity.rs:55-67)
    float2 R[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) R[j] = make_float2(0.f, 0.f);
    for (int yy = y0; yy < y1; ++yy)
        for (int xx = x0; xx < x1; ++xx) {
            const float2 s = on ? imgs[(long long)c * npix + (long long)yy * nx + xx] : make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const float2 sj = shfl2(s, j);
                R[j].x += s.x * sj.x + s.y * sj.y;   // s_c conj(s_j)
                R[j].y += s.y * sj.x - s.x * sj.y;
            }
        }
    // power iteration from the centre voxel's coil vector (sensitivity.rs:69-112)
    float2 v = on ? imgs[(long long)c * npix + warp] : make_float2(0.f, 0.f);
    const float n0 = wsum(v.x * v.x + v.y * v.y);
    if (n0 == 0.f) v = make_float2(c == 0 ? 1.f : 0.f, 0.f);
    else {
        const float inv = 1.0f / sqrtf(n0);
        v = make_float2(v.x * inv, v.y * inv);
    }
    float lam = 0.f;
    for (int it = 0; it < power_iters; ++it) {
        float2 w = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float2 vj = shfl2(v, j);
            w.x += R[j].x * vj.x - R[j].y * vj.y;
            w.y += R[j].x * vj.y + R[j].y * vj.x;
        }
        if (!on) w = make_float2(0.f, 0.f);
        const float nrm = sqrtf(wsum(w.x * w.x + w.y * w.y));
        if (nrm < 1e-20f) break;
        const float inv = 1.0f / nrm;
        v = make_float2(w.x * inv, w.y * inv);
        lam = nrm;
    }
    // phase fix: the first coil of largest magnitude becomes real positive
    // (sensitivity.rs:114-131)
    float m = on ? sqrtf(v.x * v.x + v.y * v.y) : -1.f;
    int im = c;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float mo = __shfl_xor_sync(0xffffffffu, m, o);
        const int io = __shfl_xor_sync(0xffffffffu, im, o);
        if (mo > m || (mo == m && io < im)) { m = mo; im = io; }
    }
    if (m > 0.f) {
        const float2 ref = shfl2(v, im);
        v = cm(v, make_float2(ref.x / m, -ref.y / m));
    }
    const float sc = sqrtf(lam);                         // sensitivity.rs:133-138
    float2 o = make_float2(v.x * sc, v.y * sc);
    if (normalise) {
        const float rss = sqrtf(wsum(on ? o.x * o.x + o.y * o.y : 0.f));
        o = rss > 0.f ? make_float2(o.x / rss, o.y / rss) : make_float2(0.f, 0.f);
    }
    if (on) maps[(long long)c * npix + warp] = o;
}

cudaError_t launch_walsh(const float2* imgs, float2* maps, int nc, int ny, int nx, int window, int power_iters,
                         int normalise, cudaStream_t st) {
    if (nc <= 0 || nc > 32) return cudaErrorInvalidValue;
    const long long warps = (long long)ny * nx;
    const long long blocks = (warps + 7) / 8;
    k_walsh<<<(unsigned)blocks, 256, 0, st>>>(imgs, maps, nc, ny, nx, window, power_iters, normalise);
    return cudaGetLastError();
}

// ------------------------------------------------ FP64 power iteration
// One column per CTA: acc = sum_c S_c^* F_y^H m F_y (S_c v) in FP64 (ky-only
// mask; F_x cancels), with the centred unitary transform written as
// D F D / sqrt(n) and a direct FP64 DFT (twiddles w^{k} = e^{-2 pi i k/n}).
__global__ void k_sense_normal_fp64(const double2* __restrict__ v, double2* __restrict__ acc,
                                    const float2* __restrict__ maps, const uint32_t* __restrict__ rowbits, int nc,
                                    int ny, int nx, const double2* __restrict__ wtab, double* __restrict__ norm2) {
    extern __shared__ double2 zs[];
    double2* u = zs;           // [ny]
    double2* U = u + ny;       // [ny]
    double2* A = U + ny;       // [ny]
    const int x = blockIdx.x;
    const long long npix = (long long)ny * nx;
    for (int i = threadIdx.x; i < ny; i += blockDim.x) A[i] = make_double2(0.0, 0.0);
    for (int c = 0; c < nc; ++c) {
        __syncthreads();
        for (int i = threadIdx.x; i < ny; i += blockDim.x) {
            const float2 s = maps[(long long)c * npix + (long long)i * nx + x];
            const double2 vv = v[(long long)i * nx + x];
            double2 t = make_double2(s.x * vv.x - s.y * vv.y, s.x * vv.y + s.y * vv.x);
            if (i & 1) t = make_double2(-t.x, -t.y);
            u[i] = t;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < ny; k += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            if ((rowbits[k >> 5] >> (k & 31)) & 1u) {
                for (int i = 0; i < ny; ++i) {
                    const double2 w = wtab[(int)(((long long)i * k) % ny)];
                    s.x += u[i].x * w.x - u[i].y * w.y;
                    s.y += u[i].x * w.y + u[i].y * w.x;
                }
            }
            U[k] = s;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ny; i += blockDim.x) {
            double2 s = make_double2(0.0, 0.0);
            for (int k = 0; k < ny; ++k) {
                const double2 w = wtab[(int)(((long long)i * k) % ny)];   // conj for the inverse
                s.x += U[k].x * w.x + U[k].y * w.y;
                s.y += U[k].y * w.x - U[k].x * w.y;
            }
            if (i & 1) s = make_double2(-s.x, -s.y);
            s.x /= ny;
            s.y /= ny;
            const float2 m = maps[(long long)c * npix + (long long)i * nx + x];
            A[i].x += m.x * s.x + m.y * s.y;   // conj(S) * s
            A[i].y += m.x * s.y - m.y * s.x;
        }
    }
    __syncthreads();
    double part = 0.0;
    for (int i = threadIdx.x; i < ny; i += blockDim.x) {
        acc[(long long)i * nx + x] = A[i];
        part += A[i].x * A[i].x + A[i].y * A[i].y;
    }
    // block sum, then one FP64 atomic per column
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(norm2, s);
    }
}

// v <- acc / sqrt(norm2)
__global__ void k_normalise_fp64(const double2* __restrict__ acc, double2* __restrict__ v, long long n,
                                 const double* __restrict__ norm2) {
    const double nn = sqrt(*norm2);
    const double inv = nn > 0.0 ? 1.0 / nn : 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        v[q] = make_double2(acc[q].x * inv, acc[q].y * inv);
}

__global__ void k_fill_fp64(double2* __restrict__ v, long long n, double val) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        v[q] = make_double2(val, 0.0);
}

cudaError_t launch_sense_power(const float2* maps, const uint32_t* rowbits, int nc, int ny, int nx, int iters,
                               double2* v, double2* acc, const double2* wtab, double* norms, cudaStream_t st) {
    const long long n = (long long)ny * nx;
    k_fill_fp64<<<148 * 4, 256, 0, st>>>(v, n, 1.0 / sqrt((double)n));
    cudaError_t e = cudaGetLastError();
    const size_t smem = sizeof(double2) * 3 * (size_t)ny;
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sense_normal_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (int it = 0; it < iters && e == cudaSuccess; ++it) {
        k_sense_normal_fp64<<<nx, 256, smem, st>>>(v, acc, maps, rowbits, nc, ny, nx, wtab, norms + it);
        k_normalise_fp64<<<148 * 4, 256, 0, st>>>(acc, v, n, norms + it);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace oks
