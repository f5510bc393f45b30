// Readout-direction DFT on the 5th-generation tensor cores (sm_100a).
//
// Rows of complex64 are transformed by a dense complex matrix W (the DFT,
// optionally centred) written as ONE real GEMM:
//   Y[m][n'] = sum_k' X[m][k'] B[n'][k'],   X viewed as [M][2n] real,
// with B[2j][2k] = c, B[2j][2k+1] = -s, B[2j+1][2k] = s, B[2j+1][2k+1] = c
// for W[k][j] = c + i s, so the FP32 accumulator row is already the
// interleaved complex64 output row.  Split precision (3xBF16): every operand
// is a = a_hi + a_lo with a_hi = bf16(a), a_lo = bf16(a - a_hi), and
//   X B ~= X_hi B_hi + X_hi B_lo + X_lo B_hi
// is accumulated in FP32 in tensor memory (the lo*lo term is below the FP32
// rounding of the sum).
//
// Kernel (persistent, one CTA per SM looping over 128 x 256 output tiles,
// 192 threads):
//   * warp 0 lane 0: TMA producer.  A (X_hi, X_lo) and B (B_hi, B_lo) tiles
//     of 64 bf16 along K (128 B = one 128-byte swizzle row) go to a 2-stage
//     shared-memory ring, completion on an mbarrier per stage;
//   * warp 1 lane 0: MMA issuer.  tcgen05.mma kind::f16 (bf16 in, f32
//     accumulate), M = 128, N = 256, K = 16 per instruction, 3 products per
//     K step, into one of two accumulators in tensor memory (all 512
//     columns); tcgen05.commit frees each stage and signals a finished tile;
//   * warps 2-5: epilogue.  tcgen05.ld of the warp's 32 TMEM lanes (= output
//     rows), scale, store, then hand the accumulator back -- so a tile's
//     epilogue overlaps the next tile's MMAs.
// Every wait is bounded (about two seconds); on time-out the kernel records
// an error in *err, lets what it issued drain, frees its tensor memory and
// returns (okscuda_tc_status reads and clears the flag).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "kernels.h"

namespace oks {
namespace tc {

constexpr int BM = 128, BN = 256, BK = 64;
constexpr int NST = 2;
constexpr int A_BYTES = BM * BK * 2;                    // 16 KB
constexpr int B_BYTES = BN * BK * 2;                    // 32 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 96 KB
constexpr int SMEM_BYTES = NST * STAGE_BYTES + 1024 + 128;
constexpr int kThreads = 192;                          // producer warp, MMA warp, 4 epilogue warps
constexpr int kEpiThreads = 128;
constexpr long long kWaitCycles = 4000000000ll;         // ~2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on phase `parity`; false (and *err set) when it ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err, int code) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            atomicExch(err, code);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128 B,
// 8-row groups 1024 B apart (stride byte offset), sm_100 descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: D f32, A/B bf16, both K-major, N = BN, M = BM.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct Epilogue {
    float* out;          // [M][ld] floats (complex64 rows viewed as real)
    long long ld;        // row stride in floats
    long long M;         // rows
    int ncols;           // real output columns stored (2 nout)
    float scale;
    // complex output column j goes to column cols[j] (cols != nullptr) or
    // col0 + j; with colbits, a column whose bit is clear in the row's mask
    // (problem m / rows_per_prob, mask (problem + mask_offset) % mask_mod) is
    // stored as zero
    const int* cols;
    int col0;
    const uint32_t* colbits;
    int col_wstride;
    int rows_per_prob;
    long long mask_offset;
    int mask_mod;
    // start gate (tests of the bounded waits only): when non-null, the CTA
    // waits at most gate_cycles for *gate != 0 before any copy or MMA is
    // issued; on time-out it records code 7 and returns without work
    const int* gate;
    long long gate_cycles;
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Persistent: CTA b takes tiles b, b + grid, ...; tile t = (m_tile, n_tile) =
// (t / n_tiles, t % n_tiles).  Two accumulators in tensor memory (2 x BN
// columns, all 512): the epilogue of one tile overlaps the MMAs of the next.
__global__ void __launch_bounds__(kThreads, 1)
k_dft_tc(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
         const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo, int nk,
         int m_tiles, int n_tiles, Epilogue ep, int* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned tile area (the 128-byte swizzle repeats every 1024 B)
    uint8_t* tiles = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    // full[NST], empty[NST], tfull[2], tempty[2], done
    uint64_t* bars = reinterpret_cast<uint64_t*>(tiles + NST * STAGE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NST + 5);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + NST);
    const uint32_t tfull0 = smem_u32(bars + 2 * NST), tempty0 = smem_u32(bars + 2 * NST + 2);
    const uint32_t done = smem_u32(bars + 2 * NST + 4);
    const int ntiles = m_tiles * n_tiles;

    if (ep.gate) {
        __shared__ int s_abort;
        if (threadIdx.x == 0) {
            const long long t0 = clock64();
            int open = *(volatile const int*)ep.gate;
            while (!open && clock64() - t0 <= ep.gate_cycles) open = *(volatile const int*)ep.gate;
            s_abort = open ? 0 : 1;
            if (!open) atomicExch(err, 7);
        }
        __syncthreads();
        if (s_abort) return;   // nothing issued, no tensor memory held
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull0 + 8 * b, 1);
            mbar_init(tempty0 + 8 * b, kEpiThreads);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)(2 * BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // ---- TMA producer: the K blocks of every tile through the ring
        long long g = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const int m_tile = t / n_tiles, n_tile = t - m_tile * n_tiles;
            for (int kb = 0; kb < nk; ++kb, ++g) {
                const int s = (int)(g % NST);
                if (g >= NST && !mbar_wait(empty0 + 8 * s, (uint32_t)((g / NST) & 1) ^ 1u, err, 1)) {
                    ok = false;
                    break;
                }
                uint8_t* st = tiles + s * STAGE_BYTES;
                const uint32_t fb = full0 + 8 * s;
                mbar_expect_tx(fb, STAGE_BYTES);
                tma_load_2d(smem_u32(st), &map_ahi, fb, kb * BK, m_tile * BM);
                tma_load_2d(smem_u32(st + A_BYTES), &map_alo, fb, kb * BK, m_tile * BM);
                tma_load_2d(smem_u32(st + 2 * A_BYTES), &map_bhi, fb, kb * BK, n_tile * BN);
                tma_load_2d(smem_u32(st + 2 * A_BYTES + B_BYTES), &map_blo, fb, kb * BK, n_tile * BN);
            }
        }
        // copies still in flight complete before the CTA may exit
        for (long long q = g - NST < 0 ? 0 : g - NST; q < g; ++q)
            mbar_wait(full0 + 8 * (int)(q % NST), (uint32_t)((q / NST) & 1), err, 2);
    } else if (threadIdx.x == 32) {
        // ---- MMA issuer
        long long g = 0;
        int li = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++li) {
            const int ab = li & 1;
            // the epilogue has drained this accumulator (two tiles ago)
            if (li >= 2 && !mbar_wait(tempty0 + 8 * ab, (uint32_t)((li >> 1) & 1) ^ 1u, err, 3)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + (uint32_t)(ab * BN);
            for (int kb = 0; kb < nk; ++kb, ++g) {
                const int s = (int)(g % NST);
                if (!mbar_wait(full0 + 8 * s, (uint32_t)((g / NST) & 1), err, 4)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_hi = smem_u32(tiles + s * STAGE_BYTES);
                const uint32_t a_lo = a_hi + A_BYTES, b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk) {
                    const uint32_t o = kk * 32;   // 16 bf16 along K inside the 128-byte row
                    mma_bf16(acc, sw128_desc(a_hi + o), sw128_desc(b_hi + o), (kb | kk) != 0);
                    mma_bf16(acc, sw128_desc(a_hi + o), sw128_desc(b_lo + o), 1u);
                    mma_bf16(acc, sw128_desc(a_lo + o), sw128_desc(b_hi + o), 1u);
                }
                mma_commit(empty0 + 8 * s);   // the stage is free once these MMAs have read it
            }
            if (ok) mma_commit(tfull0 + 8 * ab);   // the tile's accumulator is complete
        }
        mma_commit(done);                          // every MMA issued above has completed
    } else if (warp >= 2) {
        // ---- epilogue: warp w owns TMEM lanes (= tile rows) 32 (w % 4) .. +31
        const int q = warp & 3;
        int li = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
            const int ab = li & 1;
            const int m_tile = t / n_tiles, n_tile = t - m_tile * n_tiles;
            const bool ok = mbar_wait(tfull0 + 8 * ab, (uint32_t)((li >> 1) & 1), err, 5);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long long row = (long long)m_tile * BM + q * 32 + lane;
            const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * BN);
            const uint32_t* rbits = nullptr;
            if (ep.colbits && row < ep.M)
                rbits = ep.colbits + ((row / ep.rows_per_prob + ep.mask_offset) % ep.mask_mod) * ep.col_wstride;
            float* orow = ep.out + row * ep.ld;
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_ld16(tl + (uint32_t)c, v);
                const int rc0 = n_tile * BN + c;   // real output column of v[0]
                if (!ok || row >= ep.M || rc0 >= ep.ncols) continue;
                if (!ep.cols && !rbits && rc0 + 16 <= ep.ncols && ((ep.ld | ep.col0) % 2) == 0) {
                    float* dst = orow + 2 * ep.col0 + rc0;
                    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
#pragma unroll
                        for (int i = 0; i < 16; i += 4)
                            *reinterpret_cast<float4*>(dst + i) = make_float4(v[i] * ep.scale, v[i + 1] * ep.scale,
                                                                             v[i + 2] * ep.scale, v[i + 3] * ep.scale);
                        continue;
                    }
                }
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    if (rc0 + i >= ep.ncols) break;
                    const int j = (rc0 + i) >> 1;
                    const int x = ep.cols ? ep.cols[j] : ep.col0 + j;
                    const bool keep = !rbits || ((__ldg(rbits + (x >> 5)) >> (x & 31)) & 1u);
                    *reinterpret_cast<float2*>(orow + 2 * x) =
                        keep ? make_float2(v[i] * ep.scale, v[i + 1] * ep.scale) : make_float2(0.f, 0.f);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(tempty0 + 8 * ab);           // this accumulator may be reused
            if (!ok) break;
        }
    }
    __syncwarp();
    // every MMA has completed before the tensor memory is released
    mbar_wait(done, 0, err, 6);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)(2 * BN)));
}

// X (complex rows, [M][ld] complex) -> hi/lo bf16 [M][kp] (real view of the
// nin gathered columns cols[a] or col0 + a, zero padded to kp reals).
__global__ void k_split_rows(const float2* __restrict__ x, long long ld, long long M, int nin,
                             const int* __restrict__ cols, int col0, int kp, __nv_bfloat162* __restrict__ hi,
                             __nv_bfloat162* __restrict__ lo) {
    const int kh = kp / 2;
    const long long total = M * (long long)kh;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = i / kh;
        const int a = (int)(i - m * kh);
        const float2 v = a < nin ? x[m * ld + (cols ? __ldg(cols + a) : col0 + a)] : make_float2(0.f, 0.f);
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        const float2 hf = __bfloat1622float2(h);
        hi[i] = h;
        lo[i] = __floats2bfloat162_rn(v.x - hf.x, v.y - hf.y);
    }
}

// ------------------------------------------------------------------ host
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// bf16 [rows][kp] row-major, box {BK, box_rows}, 128-byte swizzle.
static bool make_map(CUtensorMap* map, const void* base, long long rows, int kp, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static uint16_t bf16_bits(float f) {   // round to nearest even
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static float bf16_float(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

int kpad(int n) { return (2 * n + BK - 1) / BK * BK; }
int npad(int n) { return (2 * n + BN - 1) / BN * BN; }

// B operand of the (centred) DFT of length n, sign -1 forward / +1 inverse,
// from the input columns in_idx (empty: all n) to the output columns out_idx
// (empty: all n): hi and lo, each [npad(nout)][kpad(nin)] bf16 (B^T,
// K-major), built in FP64.
void dft_matrix_split(int n, int sign, int centred, const std::vector<int>& in_idx, const std::vector<int>& out_idx,
                      std::vector<uint16_t>* hi, std::vector<uint16_t>* lo) {
    const int nin = in_idx.empty() ? n : (int)in_idx.size();
    const int nout = out_idx.empty() ? n : (int)out_idx.size();
    const int kp = kpad(nin), np = npad(nout);
    hi->assign((size_t)np * kp, 0);
    lo->assign((size_t)np * kp, 0);
    const long long h = n / 2;
    const double two_pi = 6.283185307179586476925286766559;
    for (int j = 0; j < nout; ++j) {
        const long long jj = out_idx.empty() ? j : out_idx[j];
        for (int k = 0; k < nin; ++k) {
            const long long kk = in_idx.empty() ? k : in_idx[k];
            long long e;
            if (centred) e = (((jj - h) * (kk - h)) % n + n) % n;   // fftshift o DFT o ifftshift
            else e = (jj * kk) % n;
            const double ang = two_pi * (double)e / n;
            const double c = std::cos(ang), s = sign * std::sin(ang);
            const double vals[4] = {c, -s, s, c};   // [2j][2k], [2j][2k+1], [2j+1][2k], [2j+1][2k+1]
            const size_t idx[4] = {(size_t)(2 * j) * kp + 2 * k, (size_t)(2 * j) * kp + 2 * k + 1,
                                   (size_t)(2 * j + 1) * kp + 2 * k, (size_t)(2 * j + 1) * kp + 2 * k + 1};
            for (int q = 0; q < 4; ++q) {
                const float f = (float)vals[q];
                const uint16_t bh = bf16_bits(f);
                (*hi)[idx[q]] = bh;
                (*lo)[idx[q]] = bf16_bits((float)((double)f - (double)bf16_float(bh)));
            }
        }
    }
}

}  // namespace tc

bool dft_tc_available() { return tc::encode_fn() != nullptr; }

size_t dft_tc_scratch_bytes(long long M, int nin) { return (size_t)M * tc::kpad(nin) * 2 * 2; }

cudaError_t launch_dft_tc(const DftTcArgs& a, cudaStream_t st) {
    using namespace tc;
    const int kp = kpad(a.nin), np = npad(a.nout);
    __nv_bfloat16* a_hi = static_cast<__nv_bfloat16*>(a.scratch);
    __nv_bfloat16* a_lo = a_hi + (size_t)a.M * kp;
    {
        const long long total = a.M * (long long)(kp / 2);
        const int threads = 256;
        const long long blocks = std::min<long long>((total + threads - 1) / threads, 148ll * 16);
        k_split_rows<<<(unsigned)blocks, threads, 0, st>>>(a.in, a.ld_in, a.M, a.nin, a.in_cols, a.in_col0, kp,
                                                           reinterpret_cast<__nv_bfloat162*>(a_hi),
                                                           reinterpret_cast<__nv_bfloat162*>(a_lo));
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    CUtensorMap m_ahi, m_alo, m_bhi, m_blo;
    if (!make_map(&m_ahi, a_hi, a.M, kp, BM) || !make_map(&m_alo, a_lo, a.M, kp, BM) ||
        !make_map(&m_bhi, a.b_hi, np, kp, BN) || !make_map(&m_blo, a.b_lo, np, kp, BN))
        return cudaErrorInvalidValue;
    e = cudaFuncSetAttribute(k_dft_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) return e;
    Epilogue ep{};
    ep.out = reinterpret_cast<float*>(a.out);
    ep.ld = 2 * a.ld_out;
    ep.M = a.M;
    ep.ncols = 2 * a.nout;
    ep.scale = a.scale;
    ep.cols = a.out_cols;
    ep.col0 = a.out_col0;
    ep.colbits = a.colbits;
    ep.col_wstride = a.col_wstride;
    ep.rows_per_prob = a.rows_per_prob > 0 ? a.rows_per_prob : 1;
    ep.mask_offset = a.mask_offset;
    ep.mask_mod = a.mask_mod > 0 ? a.mask_mod : 1;
    ep.gate = a.gate;
    ep.gate_cycles = a.gate_cycles;
    const int n_tiles = np / BN, m_tiles = (int)((a.M + BM - 1) / BM);
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm < 1) nsm = 148;
    }
    // persistent: one CTA per SM (its shared memory and all 512 TMEM columns)
    const int grid = std::min(n_tiles * m_tiles, nsm);
    k_dft_tc<<<grid, kThreads, SMEM_BYTES, st>>>(m_ahi, m_alo, m_bhi, m_blo, kp / BK, m_tiles, n_tiles, ep, a.err);
    return cudaGetLastError();
}

}  // namespace oks
