// Host-side launch interface of the sm_100a kernels (no device code here).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_dev.cuh"

namespace oks {

// Device copy of one FFT length's plan: the FftPlan (by value) plus its
// twiddle and root tables in global memory.
struct DevPlan {
    FftPlan plan;
    float2* tw = nullptr;      // plan.tw_total entries
    float2* roots = nullptr;   // sum of radices entries
    int roots_total = 0;
};

// ky row mask passed by value as a kernel parameter (no per-call upload).
constexpr int kMaxMaskRows = 4096;
struct RowBits {
    uint32_t w[kMaxMaskRows / 32];
};
__host__ __device__ inline bool row_on(const RowBits& b, int r) { return (b.w[r >> 5] >> (r & 31)) & 1u; }

// Batched transform of contiguous rows: out[row][k] for nrows rows of length n.
struct RowXformArgs {
    const float2* in;
    float2* out;
    long long nrows;
    long long ld_in, ld_out;
    int sign;            // -1 forward, +1 inverse (unnormalised)
    int centred;         // reference ifftshift -> DFT -> fftshift (any n)
    float scale;
    int rows_per_prob;   // row index r within a problem is row % rows_per_prob
    int rowsign;         // multiply row r by (-1)^r
    int use_keep;        // rows r with row_on(keep, r) == false are zero
};
cudaError_t launch_row_xform(const RowXformArgs& a, const RowBits& keep, const DevPlan& pl,
                             cudaStream_t st);

// Batched transform along y of [nprob][ny][nx] in place.
struct ColXformArgs {
    float2* data;
    long long nprob;
    int ny, nx;
    long long prob_stride;
    int sign, centred;
    float scale;
};
cudaError_t launch_col_xform(const ColXformArgs& a, const DevPlan& pl, cudaStream_t st);

// Fused per-column-pair FISTA for ky-only masks (see k_fista_col).
struct FistaColArgs {
    const float2* ytil;       // prepared hybrid data y' ([ny][nx] per problem)
    long long prob_stride;
    float minv;               // m' = 1/ny on sampled rows (RowBits), 0 elsewhere
    float2* xout;             // coil images x ([ny][nx] per problem); may alias ytil
    long long out_stride;
    int ny, nx, iters;
    float lambda;
    const float* alpha;       // [iters] FISTA momentum weights
    long long nprob;
};
cudaError_t launch_fista_col(const FistaColArgs& a, const RowBits& mask, const DevPlan& pl,
                             cudaStream_t st);

// RSS over coils with centre crop: out[(y)][(x)] = sqrt(sum_c |in_c[y0+y][x0+x]|^2)
struct RssArgs {
    const float2* coils;     // coil c at coils + c * coil_stride, [ny][nx]
    long long coil_stride;
    int nc, ny, nx;
    int y0, x0, ty, tx;      // crop window
    float* out;              // [ty][tx]
};
cudaError_t launch_rss(const RssArgs& a, cudaStream_t st);

// Haar primitives on [nprob][ny][nx]
cudaError_t launch_haar(const float2* in, float2* out, long long nprob, int ny, int nx, int inverse,
                        cudaStream_t st);
cudaError_t launch_soft_threshold(float2* data, long long nprob, int ny, int nx, float lambda,
                                  cudaStream_t st);

}  // namespace oks
