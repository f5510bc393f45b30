// Register-resident fused column FISTA for ky-only masks (sm_100a).
//
// Same mathematics as k_fista_col (k_cs.cu header comment): one column pair
// (2j, 2j+1) of one coil runs every FISTA iteration on chip.  Here the state
// lives in registers:
//   * a group of T threads owns one column pair; thread t holds the elements
//     q = t + TA*e (e < E = 2N/TA) of the interleaved pair, q = 2*row + col,
//     for x~, z~, y' and the work vector (TA = active threads, T = TA rounded
//     up to whole warps);
//   * every Stockham stage reads its inputs at rows i + j N/R, which for the
//     first forward stage and the fused middle are exactly the thread's own
//     registers (R | E); intermediate stages exchange through shared memory
//     with an XOR-swizzled index (padi in reg_fft.cuh) that keeps the
//     strided writes nearly conflict-free;
//   * the last forward stage, the data residual and the first inverse stage
//     (same radix) run back to back in registers;
//   * the 2x2 Haar blocks pair q^1 (column) and q^2 (row): two xor-shuffle
//     Hadamard steps forward, two back.
// Only y' in and the coil image out touch global memory.
#include <cuda_runtime.h>

#include "reg_fft.cuh"

namespace oks {
namespace reg {

// Resident CTAs per SM the column engine is compiled for: at least 12 warps
// (the register budget per thread follows from it), except for the E = 16
// plans, whose 16 elements per thread would spill under that budget.
template <class P>
constexpr int col_min_blocks() {
    constexpr int threads = P::T * (P::T == 32 ? 4 : 1);
    return P::E >= 16 ? 1 : (12 * 32 + threads - 1) / threads;
}

template <class P>
__global__ void __launch_bounds__(P::T * (P::T == 32 ? 4 : 1), col_min_blocks<P>())
k_fista_col_reg(FistaColArgs a, const float2* __restrict__ gtw, const float2* __restrict__ groots, int roots_total) {
    constexpr int N = P::N, E = P::E, TA = P::TA, T = P::T;
    constexpr int G = (T == 32) ? 4 : 1;                 // groups (column pairs) per CTA
    constexpr int NTW = Tw<P>::total();
    extern __shared__ float2 sm[];
    float2* TW = sm;
    float2* RT = TW + NTW;
    const int g = threadIdx.x / T;
    const int t = threadIdx.x % T;
    float2* A = RT + roots_total + g * 2 * P::SMEM_X;
    float2* B = A + P::SMEM_X;
    for (int q = threadIdx.x; q < NTW; q += blockDim.x) TW[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    __syncthreads();

    const long long unit = (long long)blockIdx.x * G + g;   // (problem, column pair)
    bool live;
    int nx, iters;
    float lam;
    const float2* yin;
    float2* xo;
    const uint32_t* mwords;
    if (a.probs) {   // batched: per-problem width, iterations, lambda, mask
        // every lane of the group, padding lanes included, runs the unit's
        // iteration count: shared-memory stages use all T lanes
        const bool uv = unit < a.nunits;
        live = uv && t < TA;
        const ColProblem pr = a.probs[uv ? find_problem(a.probs, a.nprob, unit) : 0];
        const int jp = uv ? (int)(unit - pr.unit0) : 0;
        nx = pr.nx;
        iters = uv ? pr.iters : 0;
        lam = pr.lambda;
        yin = pr.y + 2 * jp;
        xo = pr.x + 2 * jp;
        mwords = a.mask.words + (long long)pr.mask * a.mask.wstride;
    } else {
        const int npairs = a.nx / 2;
        live = unit < (long long)a.nprob * npairs && t < TA;
        const long long b = live ? unit / npairs : 0;
        const int jp = live ? (int)(unit - b * npairs) : 0;
        nx = a.nx;
        iters = a.iters;
        lam = a.lambda;
        yin = a.ytil + b * a.prob_stride + 2 * jp;
        xo = a.xout + b * a.out_stride + 2 * jp;
        mwords = a.mask.words + (b % a.mask.mod) * a.mask.wstride;
    }

    float2 y[E], x[E], z[E], w[E];
    uint32_t mb = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int q = t + TA * e;
        const int r = q >> 1;
        y[e] = live ? yin[(long long)r * nx + (q & 1)] : make_float2(0.f, 0.f);
        if (live && ((__ldg(mwords + (r >> 5)) >> (r & 31)) & 1u)) mb |= 1u << e;
    }
    const float minv = a.minv;
    // x~0 = z~0 = F^H (m' y')
#pragma unroll
    for (int e = 0; e < E; ++e) w[e] = ((mb >> e) & 1u) ? y[e] * minv : make_float2(0.f, 0.f);
    inverse<P>(w, A, B, TW, RT, t);
#pragma unroll
    for (int e = 0; e < E; ++e) { x[e] = w[e]; z[e] = w[e]; }

    const bool col1 = (t & 1) != 0, row1 = (t & 2) != 0;
    for (int it = 0; it < iters; ++it) {
        group_sync<P>();
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = z[e];
        forward<P>(w, A, B, TW, RT, t);
        // the last forward stage leaves element b + j*(E/R) = row i + j N/R,
        // f = t + TA*b, i = f >> 1: q = t + TA*(b + j E/R), the state layout,
        // so y and mb line up with w
#pragma unroll
        for (int e = 0; e < E; ++e)
            w[e] = ((mb >> e) & 1u) ? (w[e] - y[e]) * minv : make_float2(0.f, 0.f);
        group_sync<P>();
        inverse<P>(w, A, B, TW, RT, t);
        const float alpha = __ldg(a.alpha + it);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            // v~ = z~ - h ; plain Haar via two Hadamard steps across q^1, q^2
            const float2 v = z[e] - w[e];
            const float2 v1 = shfl_xor2(v, 1);
            const float2 u = col1 ? (v1 - v) : (v + v1);
            const float2 u2 = shfl_xor2(u, 2);
            float2 c = (row1 ? (u2 - u) : (u + u2)) * 0.5f;
            // this thread holds LL (0,0), HL (0,1), LH (1,0) or HH (1,1) of the
            // modulated image; (1,0) is the demodulated image's LL: untouched
            if (!(row1 && !col1)) c = shrink_c(c, lam);
            const float2 c1 = shfl_xor2(c, 1);
            const float2 s = col1 ? (c1 - c) : (c + c1);
            const float2 s2 = shfl_xor2(s, 2);
            const float2 xn = (row1 ? (s2 - s) : (s + s2)) * 0.5f;
            z[e] = xn + (xn - x[e]) * alpha;
            x[e] = xn;
        }
    }
    if (live) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            const int r = q >> 1;
            float2 v = x[e];
            if (r & 1) v = make_float2(-v.x, -v.y);
            xo[(long long)r * nx + (q & 1)] = v;
        }
    }
}

// ------------------------------------------- 2-D-mask engine, register form
// Same passes as k_fista2d.cu (see its header), one column pair (column
// pass) or one row pair (row pass) per thread group, data in registers.
// Column pass: element q = 2*row + col of the pair; the FFT runs along y.
template <class P, int MINB>
__global__ void __launch_bounds__(P::T * (P::T == 32 ? 4 : 1), MINB)
k2d_col_reg(Fista2dArgs a, int mode, const float2* __restrict__ gtw, const float2* __restrict__ groots,
            int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T;
    constexpr int G = (T == 32) ? 4 : 1;
    constexpr int NTW = Tw<P>::total();
    extern __shared__ float2 sm[];
    float2* TW = sm;
    float2* RT = TW + NTW;
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    float2* A = RT + roots_total + g * 2 * P::SMEM_X;
    float2* B = A + P::SMEM_X;
    for (int q = threadIdx.x; q < NTW; q += blockDim.x) TW[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    pdl_wait();                                       // the previous pass's S is complete
    pdl_trigger();
    __syncthreads();
    const int nx = a.nx, npairs = nx / 2;
    const bool live = t < TA;
    const float minv = a.minv, ysc = a.ysc;
    if ((a.prefetch & 1) && a.separable) {
        // Software-pipelined form: while a unit's transforms run, the loads
        // of the group's next sampled unit are in flight (cp.async into this
        // thread's own shared-memory slots, so no barrier guards them).
        float2* PS = RT + roots_total + G * 2 * P::SMEM_X + g * 2 * E * T;   // [E][T] S, then [E][T] y
        float2* PY = PS + E * T;
        const long long total = a.nprob * npairs, stride = (long long)gridDim.x * G;
        auto next_unit = [&](long long u) {
            for (; u < total; u += stride) {
                const long long p = u / npairs;
                const int x0 = 2 * (int)(u - p * npairs);
                const long long mi = (p + a.mask_offset) % a.mask_mod;
                if ((__ldg(a.colbits + mi * a.col_wstride + (x0 >> 5)) >> (x0 & 31)) & 3u) break;
            }
            return u;
        };
        auto issue = [&](long long u) {
            const long long p = u / npairs;
            const int x0 = 2 * (int)(u - p * npairs);
            const long long mi = (p + a.mask_offset) % a.mask_mod;
            const uint32_t cpair = (__ldg(a.colbits + mi * a.col_wstride + (x0 >> 5)) >> (x0 & 31)) & 3u;
            const uint32_t* __restrict__ rb = a.rowbits + mi * a.row_wstride;
            const float2* y = a.y + p * a.y_stride;
            const float2* S = a.S + p * a.st_stride;
            uint32_t mb = 0;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const int r = q >> 1;
                const long long off = (long long)r * nx + x0 + (q & 1);
                const bool m = live && (((__ldg(rb + (r >> 5)) >> (r & 31)) & (cpair >> (q & 1)) & 1u) != 0);
                if (m) mb |= 1u << e;
                if (!OKS_IN(e * T + t, E * T, OKS_B_STAGE)) continue;
                cp_async8(PY + e * T + t, m ? y + off : y, m ? 8u : 0u);
                if (mode) cp_async8(PS + e * T + t, live ? S + off : S, live ? 8u : 0u);
            }
            cp_async_commit();
            return mb;
        };
        long long u = next_unit((long long)blockIdx.x * G + g);
        uint32_t mb_next = u < total ? issue(u) : 0u;
        while (u < total) {
            const long long cur = u;
            const uint32_t mb = mb_next;
            cp_async_wait_all();
            const long long p = cur / npairs;
            const int x0 = 2 * (int)(cur - p * npairs);
            float2 w[E], yv[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const int r = q >> 1, x = x0 + (q & 1);
                yv[e] = PY[e * T + t] * (((r + x) & 1) ? -ysc : ysc);
                w[e] = mode ? PS[e * T + t] : (((mb >> e) & 1u) ? yv[e] * minv : make_float2(0.f, 0.f));
            }
            u = next_unit(cur + stride);
            if (u < total) mb_next = issue(u);   // in flight during the transforms below
            group_sync<P>();                     // the previous unit's last stage has read A/B
            if (mode) {
                forward<P>(w, A, B, TW, RT, t);
#pragma unroll
                for (int e = 0; e < E; ++e)
                    w[e] = ((mb >> e) & 1u) ? (w[e] - yv[e]) * minv : make_float2(0.f, 0.f);
                group_sync<P>();
            }
            inverse<P>(w, A, B, TW, RT, t);
            if (live) {
                float2* __restrict__ S = a.S + p * a.st_stride;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int q = t + TA * e;
                    S[(long long)(q >> 1) * nx + x0 + (q & 1)] = w[e];
                }
            }
        }
        cp_async_wait_all();
        return;
    }
    // persistent: the tables above are loaded once, units are grid-strided
    for (long long unit = (long long)blockIdx.x * G + g; unit < a.nprob * npairs;
         unit += (long long)gridDim.x * G) {
        const long long p = unit / npairs;
        const int x0 = 2 * (int)(unit - p * npairs);
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* cb = a.colbits + mi * a.col_wstride;
        const uint32_t cpair = (__ldg(cb + (x0 >> 5)) >> (x0 & 31)) & 3u;
        if (cpair == 0) continue;   // neither column sampled: S there reads as 0
        const float2* __restrict__ y = a.y + p * a.y_stride;
        const uint8_t* __restrict__ mk = a.mask + mi * a.mask_stride;
        const uint32_t* __restrict__ rb = a.rowbits + mi * a.row_wstride;
        float2* __restrict__ S = a.S + p * a.st_stride;
        float2 w[E], yv[E];
        uint32_t mb = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            const int r = q >> 1, x = x0 + (q & 1);
            const long long off = (long long)r * nx + x;
            // separable masks: row bit and column bit (both L1-resident)
            // instead of a byte of the mask per element
            const bool m = live && (a.separable ? (((__ldg(rb + (r >> 5)) >> (r & 31)) & (cpair >> (q & 1)) & 1u) != 0)
                                                : mk[off] != 0);
            yv[e] = m ? y[off] * (((r + x) & 1) ? -ysc : ysc) : make_float2(0.f, 0.f);
            if (m) mb |= 1u << e;
            w[e] = mode ? (live ? S[off] : make_float2(0.f, 0.f)) : (m ? yv[e] * minv : make_float2(0.f, 0.f));
        }
        group_sync<P>();                     // the previous unit's last stage has read A/B
        if (mode) {
            forward<P>(w, A, B, TW, RT, t);
#pragma unroll
            for (int e = 0; e < E; ++e) w[e] = ((mb >> e) & 1u) ? (w[e] - yv[e]) * minv : make_float2(0.f, 0.f);
            group_sync<P>();
        }
        inverse<P>(w, A, B, TW, RT, t);
        if (live) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                S[(long long)(q >> 1) * nx + x0 + (q & 1)] = w[e];
            }
        }
    }
}

// Row pass: element q = 2*x + r of the row pair (r = which row), the FFT
// runs along x; lane bit 0 pairs the rows, lane bit 1 the columns.
template <class P, int MINB>
__global__ void __launch_bounds__(P::T * (P::T == 32 ? 4 : 1), MINB)
k2d_row_reg(Fista2dArgs a, int mode, int it, const float2* __restrict__ gtw, const float2* __restrict__ groots,
            int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T, N = P::N;
    constexpr int G = (T == 32) ? 4 : 1;
    constexpr int NTW = Tw<P>::total();
    extern __shared__ float2 sm[];
    float2* TW = sm;
    float2* RT = TW + NTW;
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    float2* A = RT + roots_total + g * 2 * P::SMEM_X;
    float2* B = A + P::SMEM_X;
    for (int q = threadIdx.x; q < NTW; q += blockDim.x) TW[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    pdl_wait();                                       // the previous pass's S, X~, Z~ are complete
    pdl_trigger();
    __syncthreads();
    const int nrp = a.ny / 2;
    const bool live = t < TA;
    const float alpha = mode ? __ldg(a.alpha + it) : 0.f;
    const float lam = a.lambda;
    const bool b0 = (t & 1) != 0, b1 = (t & 2) != 0;
    const long long total = a.nprob * nrp, stride = (long long)gridDim.x * G;
    // pipelined form (a.prefetch bit 1): the next unit's S is copied
    // (cp.async) into this thread's own shared-memory slots while the current
    // unit's transforms run; Z~ and X~, needed only after the inverse
    // transform, are loaded directly
    float2* PF = RT + roots_total + G * 2 * P::SMEM_X + g * E * T;   // [E][T] S
    auto issue = [&](long long u) {
        const long long p = u / nrp;
        const int r0 = 2 * (int)(u - p * nrp);
        const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
        const long long base = p * a.st_stride + (long long)r0 * N;
        const float2* S = a.S + base;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            const int x = q >> 1;
            const long long off = (long long)(q & 1) * N + x;
            const bool on = live && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u);
            if (OKS_IN(e * T + t, E * T, OKS_B_STAGE)) cp_async8(PF + e * T + t, on ? S + off : S, on ? 8u : 0u);
        }
        cp_async_commit();
    };
    const bool pf = (a.prefetch & 2) != 0;
    if (pf && (long long)blockIdx.x * G + g < total) issue((long long)blockIdx.x * G + g);
    for (long long unit = (long long)blockIdx.x * G + g; unit < total; unit += stride) {
        const long long p = unit / nrp;
        const int r0 = 2 * (int)(unit - p * nrp);
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* cb = a.colbits + mi * a.col_wstride;
        const long long base = p * a.st_stride + (long long)r0 * N;
        float2* __restrict__ S = a.S + base;
        float2* __restrict__ X = a.X + base;
        float2* __restrict__ Z = a.Z + base;
        // every global load of the unit is issued before any store
        float2 w[E], zo[E], xo[E];
        uint32_t cm = 0;                       // column sampled, per element
        if (pf) {
            cp_async_wait_all();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const int x = q >> 1;
                const long long off = (long long)(q & 1) * N + x;
                if (live && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u)) cm |= 1u << e;
                w[e] = PF[e * T + t];
                zo[e] = (mode && live) ? Z[off] : make_float2(0.f, 0.f);
                xo[e] = (mode && live) ? X[off] : make_float2(0.f, 0.f);
            }
            if (unit + stride < total) issue(unit + stride);   // in flight during the transforms below
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const int x = q >> 1;
                const long long off = (long long)(q & 1) * N + x;
                const bool on = live && ((cb[x >> 5] >> (x & 31)) & 1u);
                if (on) cm |= 1u << e;
                w[e] = on ? S[off] : make_float2(0.f, 0.f);
                zo[e] = (mode && live) ? Z[off] : make_float2(0.f, 0.f);
                xo[e] = (mode && live) ? X[off] : make_float2(0.f, 0.f);
            }
        }
        group_sync<P>();                       // the previous unit's last stage has read A/B
        inverse<P>(w, A, B, TW, RT, t);
        if (mode == 0) {
            if (live) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int q = t + TA * e;
                    const long long off = (long long)(q & 1) * N + (q >> 1);
                    X[off] = w[e];
                    Z[off] = w[e];
                }
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const long long off = (long long)(q & 1) * N + (q >> 1);
                const float2 v = zo[e] - w[e];
                const float2 v1 = shfl_xor2(v, 1);
                const float2 u = b0 ? (v1 - v) : (v + v1);
                const float2 u2 = shfl_xor2(u, 2);
                float2 c = (b1 ? (u2 - u) : (u + u2)) * 0.5f;
                // (row-difference, column-difference) band of the modulated
                // image is the demodulated image's LL: untouched
                if (!(b0 && b1)) c = shrink_c(c, lam);
                const float2 c1 = shfl_xor2(c, 1);
                const float2 s = b0 ? (c1 - c) : (c + c1);
                const float2 s2 = shfl_xor2(s, 2);
                const float2 xn = (b1 ? (s2 - s) : (s + s2)) * 0.5f;
                const float2 zn = xn + (xn - xo[e]) * alpha;
                if (live) {
                    X[off] = xn;
                    Z[off] = zn;
                }
                w[e] = zn;
            }
        }
        group_sync<P>();
        forward<P>(w, A, B, TW, RT, t);
        if (live) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (!((cm >> e) & 1u)) continue;   // only sampled columns of S are read back
                const int q = t + TA * e;
                S[(long long)(q & 1) * N + (q >> 1)] = w[e];
            }
        }
    }
    if (pf) cp_async_wait_all();
}

// Row pass with bulk-copy staging (a.prefetch bit 2): one thread of each
// group copies the group's next row pair of S, Z~ and X~ (three contiguous
// 2 nx complex64 spans) into a shared-memory staging buffer with
// cp.async.bulk (no multicast), completing on an mbarrier, while the group
// transforms the current row pair; the group reads the staged values into
// registers, releases the buffer and issues the next copies.  The loads
// then cost no issue slots and no registers while they are in flight.
// Every mbarrier wait is bounded (about one second of clock cycles): on
// time-out the group records code 8 in *a.err, waits (bounded again) for
// the copy in flight and leaves the loop; the decision is uniform per group.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bar_init1(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
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
__device__ __forceinline__ bool bar_wait_bounded(uint32_t bar, uint32_t parity, long long cycles) {
    if (bar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!bar_try(bar, parity))
        if (clock64() - t0 > cycles) return false;
    return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// true when pred holds in any thread of the group (a warp, or the whole CTA)
template <class P>
__device__ __forceinline__ bool group_any(bool pred) {
    if constexpr (P::T == 32) return __any_sync(0xffffffffu, pred);
    else return __syncthreads_or(pred) != 0;
}
constexpr long long kRowWaitCycles = 2000000000ll;   // about one second at 1.9 GHz

template <class P, int MINB>
__global__ void __launch_bounds__(P::T * (P::T == 32 ? 4 : 1), MINB)
k2d_row_tma(Fista2dArgs a, int mode, int it, const float2* __restrict__ gtw, const float2* __restrict__ groots,
            int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T, N = P::N;
    constexpr int G = (T == 32) ? 4 : 1;
    constexpr int NTW = Tw<P>::total();
    static_assert(G == 1 || T == 32, "groups are warps or the whole CTA");
    extern __shared__ __align__(16) float2 sm[];
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    float2* STG = sm + (size_t)g * 6 * N;             // [S row pair | Z~ row pair | X~ row pair]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + (size_t)G * 6 * N);
    float2* TW = sm + (size_t)G * 6 * N + G;
    float2* RT = TW + NTW;
    float2* A = RT + roots_total + g * 2 * P::SMEM_X;
    float2* B = A + P::SMEM_X;
    for (int q = threadIdx.x; q < NTW; q += blockDim.x) TW[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    const uint32_t bar = smem_addr(&bars[g]);
    if (t == 0) {
        bar_init1(bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int nrp = a.ny / 2;
    const bool live = t < TA;
    const float alpha = mode ? __ldg(a.alpha + it) : 0.f;
    const float lam = a.lambda;
    const bool b0 = (t & 1) != 0, b1 = (t & 2) != 0;
    const long long total = a.nprob * nrp, stride = (long long)gridDim.x * G;
    constexpr uint32_t kPair = 2u * N * sizeof(float2);   // bytes of one row pair (a multiple of 16)
    auto issue = [&](long long u) {                         // thread 0 of the group
        const long long p = u / nrp;
        const int r0 = 2 * (int)(u - p * nrp);
        const long long base = p * a.st_stride + (long long)r0 * N;
        bar_expect_tx(bar, mode ? 3 * kPair : kPair);
        bulk_g2s(STG, a.S + base, kPair, bar);
        if (mode) {
            bulk_g2s(STG + 2 * N, a.Z + base, kPair, bar);
            bulk_g2s(STG + 4 * N, a.X + base, kPair, bar);
        }
    };
    uint32_t phase = 0;
    long long unit = (long long)blockIdx.x * G + g;
    if (t == 0 && unit < total) issue(unit);
    for (; unit < total; unit += stride) {
        const bool ok = bar_wait_bounded(bar, phase & 1u, kRowWaitCycles);
        if (group_any<P>(!ok)) {
            if (t == 0) {
                atomicExch(a.err, 8);
                bar_wait_bounded(bar, phase & 1u, kRowWaitCycles);   // the copy in flight lands first
            }
            break;
        }
        ++phase;
        const long long p = unit / nrp;
        const int r0 = 2 * (int)(unit - p * nrp);
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* cb = a.colbits + mi * a.col_wstride;
        const long long base = p * a.st_stride + (long long)r0 * N;
        float2* __restrict__ S = a.S + base;
        float2* __restrict__ X = a.X + base;
        float2* __restrict__ Z = a.Z + base;
        float2 w[E], zo[E], xo[E];
        uint32_t cm = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            const int x = q >> 1;
            const int off = (q & 1) * N + x;
            const bool on = live && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u) && OKS_IN(off, 2 * N, OKS_B_STAGE);
            if (on) cm |= 1u << e;
            w[e] = on ? STG[off] : make_float2(0.f, 0.f);
            zo[e] = (mode && live) ? STG[2 * N + off] : make_float2(0.f, 0.f);
            xo[e] = (mode && live) ? STG[4 * N + off] : make_float2(0.f, 0.f);
        }
        group_sync<P>();                     // staging read by the group; the last unit's final stage has read A/B
        if (t == 0 && unit + stride < total) issue(unit + stride);
        inverse<P>(w, A, B, TW, RT, t);
        if (mode == 0) {
            if (live) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int q = t + TA * e;
                    const long long off = (long long)(q & 1) * N + (q >> 1);
                    X[off] = w[e];
                    Z[off] = w[e];
                }
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e;
                const long long off = (long long)(q & 1) * N + (q >> 1);
                const float2 v = zo[e] - w[e];
                const float2 v1 = shfl_xor2(v, 1);
                const float2 u = b0 ? (v1 - v) : (v + v1);
                const float2 u2 = shfl_xor2(u, 2);
                float2 c = (b1 ? (u2 - u) : (u + u2)) * 0.5f;
                if (!(b0 && b1)) c = shrink_c(c, lam);   // the demodulated image's LL band: untouched
                const float2 c1 = shfl_xor2(c, 1);
                const float2 s2v = b0 ? (c1 - c) : (c + c1);
                const float2 s2 = shfl_xor2(s2v, 2);
                const float2 xn = (b1 ? (s2 - s2v) : (s2v + s2)) * 0.5f;
                const float2 zn = xn + (xn - xo[e]) * alpha;
                if (live) {
                    X[off] = xn;
                    Z[off] = zn;
                }
                w[e] = zn;
            }
        }
        group_sync<P>();
        forward<P>(w, A, B, TW, RT, t);
        if (live) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (!((cm >> e) & 1u)) continue;   // only sampled columns of S are read back
                const int q = t + TA * e;
                S[(long long)(q & 1) * N + (q >> 1)] = w[e];
            }
        }
    }
}

// ------------------------------------------- SENSE mode, register form
// One image per slice: g = sum_c S_c^* F_y^H m (F_y (S_c z~) - y'_c) per
// column pair (ky-only mask; maps are diagonal, so they commute with the
// row modulation), v~ = z~ - g / L, prox with lambda / L, momentum.  Maps
// and y'_c are streamed from L2 every iteration; x~, z~, g stay in registers.
template <class P>
__global__ void __launch_bounds__(P::T * (P::T == 32 ? 4 : 1))
k_sense_col_reg(SenseArgs a, const float2* __restrict__ gtw, const float2* __restrict__ groots, int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T;
    constexpr int G = (T == 32) ? 4 : 1;
    constexpr int NTW = Tw<P>::total();
    extern __shared__ float2 sm[];
    float2* TW = sm;
    float2* RT = TW + NTW;
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    float2* A = RT + roots_total + g * 2 * P::SMEM_X;
    float2* B = A + P::SMEM_X;
    for (int q = threadIdx.x; q < NTW; q += blockDim.x) TW[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    __syncthreads();
    const int nx = a.nx, npairs = nx / 2;
    const long long unit = (long long)blockIdx.x * G + g;
    if (unit >= npairs) return;
    const int x0 = 2 * (int)unit;
    const bool live = t < TA;
    const long long npix = (long long)a.ny * nx;
    const float minv = a.minv;
    uint32_t mb = 0;
    long long offs[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int q = t + TA * e;
        const int r = q >> 1;
        offs[e] = (long long)r * nx + x0 + (q & 1);
        if (live && ((__ldg(a.mask.words + (r >> 5)) >> (r & 31)) & 1u)) mb |= 1u << e;
    }
    float2 x[E], z[E], gr[E], w[E], s[E];
    // atb = sum_c S_c^* F^H (m' y'_c)
#pragma unroll
    for (int e = 0; e < E; ++e) gr[e] = make_float2(0.f, 0.f);
    for (int c = 0; c < a.nc; ++c) {
        const float2* yc = a.ytil + c * npix;
        const float2* sc = a.maps + c * npix;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            w[e] = ((mb >> e) & 1u) ? yc[offs[e]] * minv : make_float2(0.f, 0.f);
            s[e] = live ? sc[offs[e]] : make_float2(0.f, 0.f);
        }
        group_sync<P>();
        inverse<P>(w, A, B, TW, RT, t);
#pragma unroll
        for (int e = 0; e < E; ++e) gr[e] = gr[e] + cmulc(w[e], s[e]);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) { x[e] = gr[e]; z[e] = gr[e]; }
    const float lam = a.lambda_l, il = a.inv_l;
    const bool col1 = (t & 1) != 0, row1 = (t & 2) != 0;
    for (int it = 0; it < a.iters; ++it) {
#pragma unroll
        for (int e = 0; e < E; ++e) gr[e] = make_float2(0.f, 0.f);
        for (int c = 0; c < a.nc; ++c) {
            const float2* yc = a.ytil + c * npix;
            const float2* sc = a.maps + c * npix;
            float2 yv[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                s[e] = live ? sc[offs[e]] : make_float2(0.f, 0.f);
                yv[e] = ((mb >> e) & 1u) ? yc[offs[e]] : make_float2(0.f, 0.f);
                w[e] = cmul(s[e], z[e]);
            }
            group_sync<P>();
            forward<P>(w, A, B, TW, RT, t);
#pragma unroll
            for (int e = 0; e < E; ++e) w[e] = ((mb >> e) & 1u) ? (w[e] - yv[e]) * minv : make_float2(0.f, 0.f);
            group_sync<P>();
            inverse<P>(w, A, B, TW, RT, t);
#pragma unroll
            for (int e = 0; e < E; ++e) gr[e] = gr[e] + cmulc(w[e], s[e]);   // S^* h
        }
        const float alpha = __ldg(a.alpha + it);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float2 v = z[e] - gr[e] * il;
            const float2 v1 = shfl_xor2(v, 1);
            const float2 u = col1 ? (v1 - v) : (v + v1);
            const float2 u2 = shfl_xor2(u, 2);
            float2 c = (row1 ? (u2 - u) : (u + u2)) * 0.5f;
            if (!(row1 && !col1)) c = shrink_c(c, lam);   // (1,0) is the demodulated LL
            const float2 c1 = shfl_xor2(c, 1);
            const float2 sv = col1 ? (c1 - c) : (c + c1);
            const float2 s2 = shfl_xor2(sv, 2);
            const float2 xn = (row1 ? (s2 - sv) : (sv + s2)) * 0.5f;
            z[e] = xn + (xn - x[e]) * alpha;
            x[e] = xn;
        }
    }
    if (live) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            float2 v = x[e];
            if ((q >> 1) & 1) v = make_float2(-v.x, -v.y);
            if (a.xout) a.xout[offs[e]] = v;
            a.mag[offs[e]] = sqrtf(v.x * v.x + v.y * v.y);
        }
    }
}

// ------------------------------------------------------------ dispatch

// Minimum resident CTAs per SM for the 12-warp occupancy form of the 2-D
// passes (a.occ = 1); the register budget per thread follows from it.
template <class P>
constexpr int occ_blocks() {
    constexpr int threads = P::T * (P::T == 32 ? 4 : 1);
    return (12 * 32 + threads - 1) / threads;
}
// The 18-warp form (a.occ = 2): a tighter register budget for more resident
// warps (the 368 column pass compiles without spills at 6 CTAs per SM).
template <class P>
constexpr int occ_blocks_hi() {
    constexpr int threads = P::T * (P::T == 32 ? 4 : 1);
    return (18 * 32 + threads - 1) / threads;
}

template <class P, int MINB>
static cudaError_t launch_2d_k(const Fista2dArgs& a, long long units, cudaStream_t st, int mode, int it, bool row) {
    constexpr int NTW = Tw<P>::total();
    constexpr int G = (P::T == 32) ? 4 : 1;
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    // the pipelined column pass (separable masks) adds each group's prefetch
    // slots for S and y, the pipelined row pass its slots for S
    // (left out where they would cost resident CTAs below MINB per SM)
    Fista2dArgs b = a;
    const size_t base_smem = sizeof(float2) * (NTW + nrt + (size_t)G * 2 * P::SMEM_X);
    const size_t pf_smem = sizeof(float2) * (size_t)G * (row ? 1 : 2) * P::E * P::T;
    int pf = row ? ((a.prefetch & 2) ? 1 : 0) : ((a.separable && (a.prefetch & 1)) ? 1 : 0);
    if (pf && MINB > 1 && (base_smem + pf_smem + 1024) * MINB > 220u * 1024u) pf = 0;
    b.prefetch = pf ? (row ? 2 : 1) : 0;   // the kernels test their own bit
    const size_t smem = base_smem + (pf ? pf_smem : 0);
    if (row && (a.prefetch & 4) && a.err) {
        // bulk-copy staging: [S | Z~ | X~] row pairs per group, one mbarrier
        // per group (an 8-byte slot), then the tables and exchange buffers
        const size_t tsmem = sizeof(float2) * ((size_t)G * 6 * P::N + G + NTW + nrt + (size_t)G * 2 * P::SMEM_X);
        const void* fn = reinterpret_cast<const void*>(k2d_row_tma<P, MINB>);
        if ((e = set_smem_attr(fn, tsmem)) != cudaSuccess) return e;
        long long grid = (units + G - 1) / G;
        if (a.persist) {
            static int per_sm = 0, nsm = 0;
            static std::mutex mu;
            std::lock_guard<std::mutex> lk(mu);
            if (!per_sm) {
                int dev = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2d_row_tma<P, MINB>, P::T * G, tsmem);
                if (per_sm < 1) per_sm = 1;
            }
            if (grid > (long long)per_sm * nsm) grid = (long long)per_sm * nsm;
        }
        k2d_row_tma<P, MINB><<<(unsigned)grid, P::T * G, tsmem, st>>>(a, mode, it, tw, rt, nrt);
        return cudaGetLastError();
    }
    if (row) e = set_smem_attr(reinterpret_cast<const void*>(k2d_row_reg<P, MINB>), smem);
    else e = set_smem_attr(reinterpret_cast<const void*>(k2d_col_reg<P, MINB>), smem);
    if (e != cudaSuccess) return e;
    long long grid = (units + G - 1) / G;
    // persistent form: every resident CTA slot once, units grid-strided
    // (the kernels accept any grid)
    if (a.persist) {
        static int per_sm[2][2] = {{0, 0}, {0, 0}}, nsm = 0;
        static std::mutex mu;
        std::lock_guard<std::mutex> lk(mu);
        if (!per_sm[row][pf]) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (row) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1][pf], k2d_row_reg<P, MINB>, P::T * G, smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0][pf], k2d_col_reg<P, MINB>, P::T * G, smem);
            if (per_sm[row][pf] < 1) per_sm[row][pf] = 1;
        }
        int per = per_sm[row][pf];
        if (row && a.row_ctas > 0 && a.row_ctas < per) per = a.row_ctas;
        if (grid > (long long)per * nsm) grid = (long long)per * nsm;
    }
    if (row)
        return launch_pass(k2d_row_reg<P, MINB>, (unsigned)grid, P::T * G, smem, st, b.pdl != 0, b, mode, it, tw, rt,
                           nrt);
    return launch_pass(k2d_col_reg<P, MINB>, (unsigned)grid, P::T * G, smem, st, b.pdl != 0, b, mode, tw, rt, nrt);
}

// The 15-warp form (a.occ = 3): between the two above (the 368 column pass
// at 5 CTAs of 96 threads per SM, 136 registers).
template <class P>
constexpr int occ_blocks_mid() {
    constexpr int threads = P::T * (P::T == 32 ? 4 : 1);
    return (15 * 32 + threads - 1) / threads;
}

template <class P>
static cudaError_t launch_2d(const Fista2dArgs& a, long long units, cudaStream_t st, int mode, int it, bool row) {
    if (a.occ == 3) return launch_2d_k<P, occ_blocks_mid<P>()>(a, units, st, mode, it, row);
    if (a.occ == 2) return launch_2d_k<P, occ_blocks_hi<P>()>(a, units, st, mode, it, row);
    if (a.occ) return launch_2d_k<P, occ_blocks<P>()>(a, units, st, mode, it, row);
    return launch_2d_k<P, 1>(a, units, st, mode, it, row);
}

template <class P>
static cudaError_t col2d(const Fista2dArgs& a, RegTables& tabs, int mode, cudaStream_t st) {
    (void)tabs;
    // the pruned 368 forms (9-12) take the iteration passes of separable
    // masks; the init pass and other masks stay on the register pass
    const bool pruned = a.col_lanes >= 9;
    if (a.col_lanes > 0 && (a.nx % 2) == 0 && (reinterpret_cast<uintptr_t>(a.S) & 15) == 0 &&
        (!pruned || (mode == 1 && a.separable && a.ny == 368)))
        return launch_fista2d_col_lanes(a, a.col_lanes, mode, st);
    return launch_2d<P>(a, a.nprob * (a.nx / 2), st, mode, 0, false);
}
template <class P>
static cudaError_t row2d(const Fista2dArgs& a, RegTables& tabs, int mode, int it, cudaStream_t st) {
    (void)tabs;
    return launch_2d<P>(a, a.nprob * (a.ny / 2), st, mode, it, true);
}


template <class P>
static cudaError_t launch_p(const FistaColArgs& a, cudaStream_t st) {
    constexpr int NTW = Tw<P>::total();
    constexpr int G = (P::T == 32) ? 4 : 1;
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * (NTW + nrt + (size_t)G * 2 * P::SMEM_X);
    e = set_smem_attr(reinterpret_cast<const void*>(k_fista_col_reg<P>), smem);
    if (e != cudaSuccess) return e;
    const long long units = a.probs ? a.nunits : a.nprob * (long long)(a.nx / 2);
    const long long grid = (units + G - 1) / G;
    k_fista_col_reg<P><<<(unsigned)grid, P::T * G, smem, st>>>(a, tw, rt, nrt);
    return cudaGetLastError();
}

}  // namespace reg

bool fista_col_reg_supported(int ny) {
    switch (ny) {
        case 128: case 192: case 256: case 320: case 368: case 384: case 512: return true;
        default: return false;
    }
}

bool fista2d_reg_supported(int n) { return fista_col_reg_supported(n) || n == 640; }

// ---------------------------------------------------------- SENSE launch
namespace reg {

template <class P>
static cudaError_t sense_p(const SenseArgs& a, cudaStream_t st) {
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    constexpr int G = (P::T == 32) ? 4 : 1;
    const size_t smem = sizeof(float2) * (Tw<P>::total() + nrt + (size_t)G * 2 * P::SMEM_X);
    e = cudaFuncSetAttribute(k_sense_col_reg<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long grid = (a.nx / 2 + G - 1) / G;
    k_sense_col_reg<P><<<(unsigned)grid, P::T * G, smem, st>>>(a, tw, rt, nrt);
    return cudaGetLastError();
}
}  // namespace reg

bool sense_reg_supported(int ny) {
    switch (ny) {
        case 128: case 192: case 256: case 320: case 368: case 384: case 512: return true;
        default: return false;
    }
}

cudaError_t launch_sense_col_reg(const SenseArgs& a, cudaStream_t st) {
    switch (a.ny) {
        case 128: return reg::sense_p<reg::S128>(a, st);
        case 192: return reg::sense_p<reg::S192>(a, st);
        case 256: return reg::sense_p<reg::S256>(a, st);
        case 320: return reg::sense_p<reg::S320>(a, st);
        case 368: return reg::sense_p<reg::S368>(a, st);
        case 384: return reg::sense_p<reg::S384>(a, st);
        case 512: return reg::sense_p<reg::S512>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

// Host twiddle tables of every register plan, in one allocation.
cudaError_t reg_tables_init(RegTables* t) {
    if (t->ready) return cudaSuccess;
    constexpr int K = 8;
    const int ns[K] = {128, 192, 256, 320, 368, 384, 512, 640};
    size_t total = 0;
    int ntw[K] = {}, nrt[K] = {};
    static float2 htw[K][4096];
    static float2 hrt[K][64];
    reg::host_tables<reg::P128>(htw[0], &ntw[0]);
    reg::host_tables<reg::P192>(htw[1], &ntw[1]);
    reg::host_tables<reg::P256>(htw[2], &ntw[2]);
    reg::host_tables<reg::P320>(htw[3], &ntw[3]);
    reg::host_tables<reg::P368>(htw[4], &ntw[4]);
    reg::host_tables<reg::P384>(htw[5], &ntw[5]);
    reg::host_tables<reg::P512>(htw[6], &ntw[6]);
    reg::host_tables<reg::P640>(htw[7], &ntw[7]);
    // roots (cos, sin)(2 pi m / R) for the odd generic radix 23
    for (int k = 0; k < K; ++k) {
        if (ns[k] == 368) {
            for (int m = 0; m < 23; ++m) {
                const double ang = 6.283185307179586476925286766559 * m / 23.0;
                hrt[k][m] = make_float2((float)cos(ang), (float)sin(ang));
            }
            nrt[k] = 23;
        } else {
            hrt[k][0] = make_float2(1.f, 0.f);
            nrt[k] = 1;
        }
        total += ntw[k] + nrt[k];
    }
    float2* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(float2) * total);
    if (e != cudaSuccess) return e;
    size_t o = 0;
    for (int k = 0; k < K; ++k) {
        e = cudaMemcpy(d + o, htw[k], sizeof(float2) * ntw[k], cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        t->tw[ns[k]] = d + o;
        o += ntw[k];
        e = cudaMemcpy(d + o, hrt[k], sizeof(float2) * nrt[k], cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        t->roots[ns[k]] = d + o;
        t->roots_n[ns[k]] = nrt[k];
        o += nrt[k];
    }
    t->base = d;
    t->ready = true;
    return cudaSuccess;
}

cudaError_t launch_fista_col_reg(const FistaColArgs& a, RegTables& tabs, cudaStream_t st) {
    (void)tabs;
    if (a.nprob <= 0 || a.nx <= 0) return cudaSuccess;
    // variant 1: the E = 8 plans (more threads per column pair, fewer registers each)
    if (a.variant == 1) {
        switch (a.ny) {
            case 192: return reg::launch_p<reg::S192>(a, st);
            case 320: return reg::launch_p<reg::V320>(a, st);
            case 256: return reg::launch_p<reg::S256>(a, st);
            case 384: return reg::launch_p<reg::S384>(a, st);
            case 512: return reg::launch_p<reg::S512>(a, st);
            default: break;
        }
    }
    switch (a.ny) {
        case 128: return reg::launch_p<reg::P128>(a, st);
        case 192: return reg::launch_p<reg::P192>(a, st);
        case 256: return reg::launch_p<reg::P256>(a, st);
        case 320: return reg::launch_p<reg::P320>(a, st);
        case 368: return reg::launch_p<reg::P368>(a, st);
        case 384: return reg::launch_p<reg::P384>(a, st);
        case 512: return reg::launch_p<reg::P512>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

int fista_col_reg_variants(int ny) {
    return (ny == 192 || ny == 256 || ny == 320 || ny == 384 || ny == 512) ? 2 : 1;
}

cudaError_t launch_fista2d_col_reg(const Fista2dArgs& a, RegTables& tabs, int mode, cudaStream_t st) {
    if (a.nprob <= 0) return cudaSuccess;
    switch (a.ny) {
        case 128: return reg::col2d<reg::P128>(a, tabs, mode, st);
        case 192: return reg::col2d<reg::P192>(a, tabs, mode, st);
        case 256: return reg::col2d<reg::P256>(a, tabs, mode, st);
        case 320: return reg::col2d<reg::P320>(a, tabs, mode, st);
        case 368: return reg::col2d<reg::P368>(a, tabs, mode, st);
        case 384: return reg::col2d<reg::P384>(a, tabs, mode, st);
        case 512: return reg::col2d<reg::P512>(a, tabs, mode, st);
        case 640: return reg::col2d<reg::P640>(a, tabs, mode, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fista2d_row_reg(const Fista2dArgs& a, RegTables& tabs, int mode, int it, cudaStream_t st) {
    if (a.nprob <= 0) return cudaSuccess;
    switch (a.nx) {
        case 128: return reg::row2d<reg::P128>(a, tabs, mode, it, st);
        case 192: return reg::row2d<reg::P192>(a, tabs, mode, it, st);
        case 256: return reg::row2d<reg::P256>(a, tabs, mode, it, st);
        case 320: return reg::row2d<reg::P320>(a, tabs, mode, it, st);
        case 368: return reg::row2d<reg::P368>(a, tabs, mode, it, st);
        case 384: return reg::row2d<reg::P384>(a, tabs, mode, it, st);
        case 512: return reg::row2d<reg::P512>(a, tabs, mode, it, st);
        case 640: return reg::row2d<reg::P640>(a, tabs, mode, it, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace oks
