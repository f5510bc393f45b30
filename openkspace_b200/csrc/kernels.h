// Host-side launch interface of the sm_100a kernels (no device code here).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "fft_dev.cuh"

namespace oks {

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device,
// size) instead of before every launch: the 2-D engine issues thousands of
// launches per call, and the host's launch rate can bound it.
inline cudaError_t set_smem_attr(const void* fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t& v = done[{fn, dev}];
    if (v >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) v = smem;
    return e;
}

// Device copy of one FFT length's plan: the FftPlan (by value) plus its
// twiddle and root tables in global memory.
struct DevPlan {
    FftPlan plan;
    float2* tw = nullptr;      // plan.tw_total entries
    float2* roots = nullptr;   // sum of radices entries
    int roots_total = 0;
};

// ky row masks on the device: mask m is `wstride` 32-bit words at
// words + m * wstride; row r is bit (r & 31) of word r >> 5.  Problem b uses
// mask (b % mod) -- e.g. b = c * nz + kz with mod = nz gives one mask per slice.
struct RowMasks {
    const uint32_t* words;
    int wstride;
    int mod;
};
__device__ __forceinline__ bool row_on(const RowMasks& m, long long prob, int r) {
    return (__ldg(m.words + (prob % m.mod) * m.wstride + (r >> 5)) >> (r & 31)) & 1u;
}

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
    int use_keep;        // rows outside the problem's row mask are zero
    RowMasks keep;
    int reg = 1;         // register-resident kernel where a plan of length n exists
    int vec16 = 0;       // set by the launcher: rows start on 16-byte boundaries
    // caller-owned device tables of the register plan (row_xform_reg_tables
    // layout); null: the tables the library builds on first use
    const float2* tables = nullptr;
    int tables_nroots = 0;
    int variant = 0;     // register kernel: 0 the default plan per length, 1 / 2 alternatives (192, 320)
};
cudaError_t launch_row_xform(const RowXformArgs& a, const DevPlan& pl, cudaStream_t st);

// Batched transform along y of [nprob][ny][nx] in place.
struct ColXformArgs {
    float2* data;
    long long nprob;
    int ny, nx;
    long long prob_stride;
    int sign, centred;
    float scale;
    int reg = 1;         // register-resident kernel where a plan of length ny exists
    int tile = 0;        // column pairs per CTA of that kernel (0: by length; 2, 4, 8)
    int lanes = 0;       // lanes-across-columns form: 0 by length, 1..4 a (width, threads) choice, -1 off
    int lanes_pf = 1;    // lanes form: 1 = next tile staged in shared memory (cp.async) during the current one
};
cudaError_t launch_col_xform(const ColXformArgs& a, const DevPlan& pl, cudaStream_t st);

// Register-resident centred transforms (k_xform_reg.cu) for the lengths with
// a register plan; even lengths only, the shifts folded into sign flips.
bool xform_reg_supported(int n);
cudaError_t launch_row_xform_reg(const RowXformArgs& a, int n, cudaStream_t st);
// Host image of the tables the register row transform of length n uses
// (RowXformArgs::tables): returns the number of float2 written to h (0 when
// n has no register plan or cap is too small), the roots count in *nroots.
int row_xform_reg_tables(int n, float2* h, int cap, int* nroots);
cudaError_t launch_col_xform_reg(const ColXformArgs& a, cudaStream_t st);

// One problem (one coil of one slice) of a batched launch with per-problem
// width, iteration count, lambda and mask (FistaColArgs::probs).
struct ColProblem {
    const float2* y;          // prepared y' [ny][nx]
    float2* x;                // coil image out [ny][nx] (may equal y)
    int nx;
    int iters;
    float lambda;
    int mask;                 // mask index into FistaColArgs::mask.words
    long long unit0;          // first (problem, column pair) unit of this problem
};

// Fused per-column-pair FISTA for ky-only masks (see k_fista_col).
struct FistaColArgs {
    const float2* ytil;       // prepared hybrid data y' ([ny][nx] per problem)
    long long prob_stride;
    float minv;               // m' = 1/ny on sampled rows, 0 elsewhere
    RowMasks mask;
    float2* xout;             // coil images x ([ny][nx] per problem); may alias ytil
    long long out_stride;
    int ny, nx, iters;
    float lambda;
    const float* alpha;       // [iters] FISTA momentum weights
    long long nprob;
    // batched form: when probs != nullptr the launch covers `nunits`
    // (problem, column pair) units of problems[0..nprob); problem p owns
    // units [probs[p].unit0, probs[p].unit0 + nx/2) and its own nx, iters,
    // lambda and mask; ytil/xout/nx/iters/lambda above are then unused
    const ColProblem* probs;
    long long nunits;
    int variant;              // register engine: 0 primary plan, 1 alternative plan where one exists
};
cudaError_t launch_fista_col(const FistaColArgs& a, const DevPlan& pl, cudaStream_t st);

// Resolves a unit of a batched launch (binary search over unit0).
__device__ __forceinline__ int find_problem(const ColProblem* probs, long long nprob, long long unit) {
    long long lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (probs[mid].unit0 <= unit) lo = mid;
        else hi = mid - 1;
    }
    return (int)lo;
}

// Register-resident column FISTA (k_fista_reg.cu) for the column lengths it
// has compile-time plans for; twiddle tables for every plan live in one
// device allocation made on first use.
struct RegTables {
    bool ready = false;
    float2* base = nullptr;
    float2* tw[1025] = {};
    float2* roots[1025] = {};
    int roots_n[1025] = {};
};
bool fista_col_reg_supported(int ny);
cudaError_t reg_tables_init(RegTables* t);
cudaError_t launch_fista_col_reg(const FistaColArgs& a, RegTables& tabs, cudaStream_t st);
int fista_col_reg_variants(int ny);   // number of register plans for this column length

// FISTA for arbitrary 2-D masks (k_fista2d.cu): state X~, Z~, S per problem.
// Launch of a 2-D pass: with pdl, as a programmatic dependent launch (the
// kernel calls pdl_wait() before it touches what the previous grid wrote).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pass(void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                               bool pdl, Args... args) {
    if (!pdl) {
        kern<<<grid, block, smem, st>>>(args...);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

struct Fista2dArgs {
    const float2* y;          // k-space [ny][nx] per problem
    long long y_stride;
    const uint8_t* mask;      // byte masks [ny][nx]; problem p uses mask p % mask_mod
    long long mask_stride;
    int mask_mod;
    long long mask_offset;    // problem p uses mask (p + mask_offset) % mask_mod
    const uint32_t* colbits;  // per mask: kx columns with any sample (ceil(nx/32) words each)
    int col_wstride;
    // every mask is separable, mask = rowbits (x) colbits: the register
    // column pass reads these bits instead of the byte masks
    const uint32_t* rowbits;  // per mask: ky rows with any sample (ceil(ny/32) words each)
    int row_wstride;
    int separable;
    float2* X;
    float2* Z;
    float2* S;
    long long st_stride;      // per-problem stride of X, Z, S
    int ny, nx;
    float ysc;                // (-1)^{ny/2 + nx/2} sqrt(ny nx)
    float minv;               // 1 / (ny nx)
    float lambda;
    const float* alpha;
    long long nprob;
    int persist;              // register passes: grid of resident CTAs, units grid-strided
    int occ;                  // register passes: 0 registers as needed, 1 at least 12 warps per SM, 2 at least 18
    int prefetch;             // register passes: next unit's loads in flight (cp.async); bit 0 column
                              // pass (separable masks), bit 1 row pass; bit 2 row pass with
                              // bulk-copy (cp.async.bulk) staging of S, Z~, X~
    int* err;                 // bounded-wait error word (bulk-copy row pass), may be null
    int pdl;                  // register passes: programmatic dependent launches (prologue overlaps the
                              // previous pass's tail)
    int row_ctas;             // > 0: the persistent row pass takes at most this many CTAs per SM
    int col_ctas;             // > 0: the pruned 368 column pass takes at most this many CTAs per SM
                              // (room for the other stream's pass on the same SM)
    int col_lanes;            // column pass in the lanes form: 0 off, else the form (1-8); 9-12
                              // the pruned 368 forms (separable masks, iteration passes)
};
cudaError_t launch_fista2d_col(const Fista2dArgs& a, const DevPlan& py, int mode, cudaStream_t st);
cudaError_t launch_fista2d_row(const Fista2dArgs& a, const DevPlan& px, int mode, int it, cudaStream_t st);
// Register-resident forms of the two passes (k_fista_reg.cu) for lengths
// with a compile-time plan (column pass: ny; row pass: nx).
bool fista2d_reg_supported(int n);
cudaError_t launch_fista2d_col_reg(const Fista2dArgs& a, RegTables& tabs, int mode, cudaStream_t st);
cudaError_t launch_fista2d_row_reg(const Fista2dArgs& a, RegTables& tabs, int mode, int it, cudaStream_t st);
// Column pass in the lanes form (k_xform_reg.cu): form 1-4 (16,32) (16,64)
// (8,64) (8,32) columns x threads per column, 5-8 the 368 forms (16,16) (8,16)
// (16,32) (8,32); 9-12 the 368 forms pruned to the sampled rows, (8,16) (8,32)
// (16,16) (16,32) (13: (8,16) with swizzled row slots; 14: the two-stage
// plan 16 · 23 with the residual fused), for separable masks and mode 1 only.
cudaError_t launch_fista2d_col_lanes(const Fista2dArgs& a, int form, int mode, cudaStream_t st);
cudaError_t launch_fista2d_demod(const float2* X, float2* out, long long nprob, int ny, int nx, long long in_stride,
                                 long long out_stride, cudaStream_t st);

// SENSE extension mode (k_sense.cu, k_fista_reg.cu).
struct SenseArgs {
    const float2* ytil;       // [nc][ny][nx] prepared y'_c (row pass output)
    const float2* maps;       // [nc][ny][nx] sensitivity maps (unit RSS)
    int nc, ny, nx, iters;
    float minv;               // 1/ny
    float lambda_l;           // lambda / L
    float inv_l;              // 1 / L
    RowMasks mask;            // the slice's row mask
    const float* alpha;
    float2* xout;             // [ny][nx] complex image, or nullptr
    float* mag;               // [ny][nx] |x|
};
bool sense_reg_supported(int ny);
cudaError_t launch_sense_col_reg(const SenseArgs& a, cudaStream_t st);
cudaError_t launch_walsh(const float2* imgs, float2* maps, int nc, int ny, int nx, int window, int power_iters,
                         int normalise, cudaStream_t st);
cudaError_t launch_sense_power(const float2* maps, const uint32_t* rowbits, int nc, int ny, int nx, int iters,
                               double2* v, double2* acc, const double2* wtab, double* norms, cudaStream_t st);

// RSS over coils with centre crop, per slice s:
//   out[s][y][x] = sqrt(sum_c |coils[c * coil_stride + s * slice_stride + (y0+y) nx + x0+x]|^2)
struct RssArgs {
    const float2* coils;
    long long coil_stride;
    int nc, ny, nx;
    int nslice;
    long long slice_stride;
    int y0, x0, ty, tx;      // crop window
    float* out;              // [nslice][ty][tx]
};
cudaError_t launch_rss(const RssArgs& a, cudaStream_t st);

// Haar primitives on [nprob][ny][nx]
cudaError_t launch_haar(const float2* in, float2* out, long long nprob, int ny, int nx, int inverse,
                        cudaStream_t st);
cudaError_t launch_soft_threshold(float2* data, long long nprob, int ny, int nx, float lambda,
                                  cudaStream_t st);

// Pinned host + device slots for small per-call uploads (see api.cu).
struct Staging {
    struct Slot {
        void* host = nullptr;
        void* dev = nullptr;
        size_t cap = 0;
        cudaEvent_t ev = nullptr;
    };
    static constexpr int kSlots = 64;   // >= requests in flight on the request server
    Slot slots[kSlots];
    int next = 0;
    // uploads of 1 MiB and more (2-D masks, large tables) take one of two
    // slots of their own, so their pinned and device buffers are allocated
    // once instead of once per ring slot
    static constexpr size_t kBig = size_t(1) << 20;
    Slot big[2];
    int next_big = 0;
    void release() {
        for (auto& s : big) {
            if (s.ev) cudaEventSynchronize(s.ev), cudaEventDestroy(s.ev);
            if (s.host) cudaFreeHost(s.host);
            if (s.dev) cudaFree(s.dev);
            s = Slot{};
        }
        for (auto& s : slots) {
            if (s.ev) cudaEventSynchronize(s.ev), cudaEventDestroy(s.ev);
            if (s.host) cudaFreeHost(s.host);
            if (s.dev) cudaFree(s.dev);
            s = Slot{};
        }
    }
};

// Tensor-core (tcgen05, split 3xBF16) row DFT (k_dft_tc.cu).
namespace tc {
int kpad(int n);   // 2n reals rounded up to the K block
int npad(int n);   // 2n reals rounded up to the N tile
void dft_matrix_split(int n, int sign, int centred, const std::vector<int>& in_idx, const std::vector<int>& out_idx,
                      std::vector<uint16_t>* hi, std::vector<uint16_t>* lo);
}  // namespace tc
bool dft_tc_available();
size_t dft_tc_scratch_bytes(long long M, int nin);
// out[m][out col j] = scale * sum_k in[m][in col k] W[k][j] for M rows.
struct DftTcArgs {
    const float2* in;
    long long ld_in;          // complex elements
    int nin;                  // input columns: in_cols[k] (nullable) or in_col0 + k
    const int* in_cols;
    int in_col0;
    float2* out;
    long long ld_out;
    int nout;                 // output columns: out_cols[j] (nullable) or out_col0 + j
    const int* out_cols;
    int out_col0;
    long long M;
    float scale;
    // optional: output columns clear in the row's mask are stored as zero
    // (row m is problem m / rows_per_prob, mask (problem + mask_offset) % mask_mod)
    const uint32_t* colbits;
    int col_wstride;
    int rows_per_prob;
    long long mask_offset;
    int mask_mod;
    const void* b_hi;         // tc::dft_matrix_split of (nin -> nout)
    const void* b_lo;
    void* scratch;            // dft_tc_scratch_bytes(M, nin)
    int* err;                 // bounded-wait error flag
    // bounded-wait test: a device word the kernel waits on (at most
    // gate_cycles) before any work; null in every production launch
    const int* gate = nullptr;
    long long gate_cycles = 0;
};
cudaError_t launch_dft_tc(const DftTcArgs& a, cudaStream_t st);
// Haar prox + momentum between the two tensor-core transforms of the 2-D
// engine's row pass (k_fista2d.cu): mode 0 sets X = Z = W; mode 1 forms
// v = Z - W, shrinks its Haar details, X' = prox, Z' = X' + alpha (X' - X).
cudaError_t launch_fista2d_prox(const Fista2dArgs& a, const float2* W, int mode, int it, cudaStream_t st);

}  // namespace oks
