// Standalone centred transforms along rows and columns, register form (sm_100a).
//
// The centred DFT of cs.rs:141-218 (ifftshift -> DFT -> fftshift, shift.rs:11-26)
// for an even length n is a plain DFT between two sign modulations:
//   out[k] = (-1)^(k + n/2) * sum_m (-1)^m x[m] w^(m k),   w = e^(-+2 pi i / n),
// since rotating the input by n/2 multiplies the DFT by (-1)^k and rotating
// the output by n/2 turns (-1)^m into a half-period shift.  The shifts are
// therefore sign flips on load and store, and the transform itself is one
// register-resident Stockham plan (reg_fft.cuh) per pair of lines.
//
// Rows (k_row_xform_reg): one thread group per row pair.  The next pair is
// copied (cp.async, 16-byte chunks, L2 only) into the group's staging buffer
// while the current pair is transformed, so HBM reads overlap the FFT.
//
// Columns (k_col_xform_reg): one CTA per tile of 2G columns x n rows, a column
// pair per thread group.  The tile arrives through the same kind of staging
// buffer in whole 2G * 8-byte row segments; results go back through the
// groups' exchange buffers so that the CTA writes whole row segments too.
#include <type_traits>

#include "reg_fft.cuh"

namespace oks {
namespace reg {

// 16-byte asynchronous global -> shared copy, cached in L2 only; src_bytes 0
// writes zeros (the source pointer must still be valid).
__device__ __forceinline__ void cp_async16(float2* dst, const float2* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}

// Exchange buffer of one group, rounded up to 16 entries: padi keeps every
// index below 2N rounded up to 16, lin16 (the first stage's output) below
// 2N + 2N/16.  LIN = false: a kernel whose transforms use padi only.
template <class P, bool LIN = true>
constexpr int xbuf() { return ((LIN ? P::LIN16_END : P::PADI_END) + 15) / 16 * 16; }

// Groups per CTA of the row kernel (warp-sized groups share a CTA).
template <class P>
constexpr int row_groups() { return P::T == 32 ? 4 : 1; }

// Register budget per thread: 64 (32 resident warps), more for plans with a
// large odd radix, whose symmetric butterfly keeps 2 (R - 1) values live:
// 128 in the row kernel, 168 in the column kernel (its groups' exchange
// buffers sit at a runtime offset, which costs address registers).
template <class P>
constexpr bool big_odd_plan() {
    for (int s = 0; s < P::S; ++s)
        if (P::R[s] % 2 == 1 && P::R[s] > 5) return true;
    return false;
}
// Minimum resident CTAs per SM for a register budget.
template <int THREADS, int REGS>
constexpr int xform_min_blocks() { return 65536 / (THREADS * REGS) < 1 ? 1 : 65536 / (THREADS * REGS); }

// A launch runs one direction, so shared memory holds only that direction's
// twiddles: forward entries [0, NF), inverse entries [NF, total).
template <class P>
constexpr int tw_half() {
    constexpr int nf = Tw<P>::fwd(P::S), ni = Tw<P>::total() - Tw<P>::fwd(P::S);
    return nf > ni ? nf : ni;
}

// Copies direction SIGN's twiddles to TWs and returns the base pointer the
// drivers index with the full table's offsets (TWs minus the skipped part, a
// compile-time offset; it stays inside the CTA's buffers, which precede TWs).
template <class P, int SIGN>
__device__ __forceinline__ const float2* load_twiddles(float2* TWs, const float2* __restrict__ gtw) {
    constexpr int NF = Tw<P>::fwd(P::S);
    constexpr int off = SIGN > 0 ? NF : 0, n = SIGN > 0 ? Tw<P>::total() - NF : NF;
    for (int q = threadIdx.x; q < n; q += blockDim.x) TWs[q] = gtw[off + q];
    return TWs - off;
}

// The transform of direction SIGN (-1 forward, +1 unnormalised inverse).
template <class P, int SIGN, bool NB = false, bool L = true>
__device__ __forceinline__ void transform(float2* w, float2* A, float2* B, const float2* TW, const float2* RT, int t) {
    if constexpr (SIGN < 0) forward<P, NB, L>(w, A, B, TW, RT, t);
    else inverse<P, NB, L>(w, A, B, TW, RT, t);
}

template <class P, int SIGN>
__global__ void __launch_bounds__(P::T * row_groups<P>(), xform_min_blocks<P::T * row_groups<P>(), big_odd_plan<P>() ? 128 : 64>())
k_row_xform_reg(RowXformArgs a, const float2* __restrict__ gtw, const float2* __restrict__ groots, int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T, N = P::N;
    constexpr int G = row_groups<P>();
    constexpr int XB = xbuf<P>();
    extern __shared__ __align__(16) float2 sm[];
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    float2* ST = sm + g * 2 * N;                    // [2][N]: the next row pair
    float2* A = sm + G * 2 * N + g * 2 * XB;
    float2* B = A + XB;
    float2* TWs = sm + G * 2 * (N + XB);
    float2* RT = TWs + tw_half<P>();
    const float2* TW = load_twiddles<P, SIGN>(TWs, gtw);
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    __syncthreads();

    const long long npairs = (a.nrows + 1) >> 1, stride = (long long)gridDim.x * G;
    const bool live = t < TA, vec = a.vec16 != 0;
    const int cs = t & 1;                            // row of the pair this thread holds
    auto row_kept = [&](long long row) {
        if (row >= a.nrows) return false;
        return !a.use_keep || row_on(a.keep, row / a.rows_per_prob, (int)(row % a.rows_per_prob));
    };
    auto issue = [&](long long u) {
        const bool k0 = row_kept(2 * u), k1 = row_kept(2 * u + 1);
        const float2* r0 = a.in + (2 * u) * a.ld_in;
        const float2* r1 = r0 + a.ld_in;
        if (vec) {
#pragma unroll
            for (int k = t; k < N; k += T) {         // N chunks of two elements
                const int c = k >= N / 2, x = 2 * (k - c * (N / 2));
                const bool on = c ? k1 : k0;
                if (OKS_IN(c * N + x + 1, 2 * N, OKS_B_STAGE))
                    cp_async16(ST + c * N + x, on ? (c ? r1 : r0) + x : a.in, on ? 16u : 0u);
            }
        } else {
#pragma unroll
            for (int k = t; k < 2 * N; k += T) {
                const int c = k >= N, x = k - c * N;
                const bool on = c ? k1 : k0;
                if (OKS_IN(c * N + x, 2 * N, OKS_B_STAGE))
                    cp_async8(ST + c * N + x, on ? (c ? r1 : r0) + x : a.in, on ? 8u : 0u);
            }
        }
        cp_async_commit();
    };
    const float sc_n2 = (a.centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    long long u = (long long)blockIdx.x * G + g;
    if (u < npairs) issue(u);
    for (; u < npairs; u += stride) {
        cp_async_wait_all();
        group_sync<P>();                             // the pair is in ST; A/B are free
        float2 w[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = (t + TA * e) >> 1;
            float2 v = (live && OKS_IN(cs * N + x, 2 * N, OKS_B_STAGE)) ? ST[cs * N + x] : make_float2(0.f, 0.f);
            if (a.centred && (x & 1)) v = make_float2(-v.x, -v.y);
            w[e] = v;
        }
        group_sync<P>();                             // ST has been read: refill it
        if (u + stride < npairs) issue(u + stride);
        transform<P, SIGN>(w, A, B, TW, RT, t);
        const long long row = 2 * u + cs;
        if (live && row < a.nrows) {
            float s = sc_n2;
            if (a.rowsign && ((row % a.rows_per_prob) & 1)) s = -s;
            float2* o = a.out + row * a.ld_out;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int k = (t + TA * e) >> 1;
                o[k] = w[e] * ((a.centred && (k & 1)) ? -s : s);
            }
        }
    }
    cp_async_wait_all();
}

template <class P, int G, int SIGN>
__global__ void __launch_bounds__(P::T * G, xform_min_blocks<P::T * G, big_odd_plan<P>() ? 168 : 64>())
k_col_xform_reg(ColXformArgs a, const float2* __restrict__ gtw, const float2* __restrict__ groots, int roots_total) {
    constexpr int E = P::E, TA = P::TA, T = P::T, N = P::N;
    constexpr int TC = 2 * G;                        // columns per tile
    constexpr int SS = TC + 2;                       // staging row stride (float2)
    constexpr int XB = xbuf<P, false>();             // padi layout throughout (transform<..., L = false>)
    constexpr int GS = 2 * XB + 2;                   // per-group stride of the A, B buffers
    static_assert(G == 2 || G == 4 || G == 8, "2, 4 or 8 column pairs per tile");
    extern __shared__ __align__(16) float2 sm[];
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    // The strides are padded by one 16-byte chunk, so that consecutive rows
    // (staging) and consecutive groups (A) start on different bank pairs:
    // a group's column reads and the CTA's row-segment reads are then
    // conflict-free, with indices linear in the element number.
    float2* ST = sm;                                 // [N][SS] staging of the next tile
    float2* AB = sm + N * SS;
    float2* A = AB + g * GS;
    float2* B = A + XB;
    float2* TWs = AB + G * GS;
    float2* RT = TWs + tw_half<P>();
    const float2* TW = load_twiddles<P, SIGN>(TWs, gtw);
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    const int ntx = (a.nx + TC - 1) / TC;
    const long long total = a.nprob * ntx;
    auto issue = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * TC;
        const float2* base = a.data + p * a.prob_stride + x0;
        for (int k = threadIdx.x; k < N * G; k += T * G) {
            const int r = k / G, j = k % G;
            const bool on = x0 + 2 * j < a.nx;       // nx is even: chunks are whole
            if (OKS_IN(r * SS + 2 * j + 1, N * SS, OKS_B_STAGE))
                cp_async16(ST + r * SS + 2 * j, on ? base + (long long)r * a.nx + 2 * j : a.data, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    const bool live = t < TA;
    const float sc_n2 = (a.centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    long long u = blockIdx.x;
    if (u < total) issue(u);
    for (; u < total; u += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();                             // tile in ST; the last tile's stores have read A
        float2 w[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e, r = q >> 1;
            float2 v = (live && OKS_IN(r * SS + 2 * g + (q & 1), N * SS, OKS_B_STAGE)) ? ST[r * SS + 2 * g + (q & 1)]
                                                                                      : make_float2(0.f, 0.f);
            if (a.centred && (r & 1)) v = make_float2(-v.x, -v.y);
            w[e] = v;
        }
        __syncthreads();                             // every group has read ST: refill it
        if (u + gridDim.x < total) issue(u + gridDim.x);
        transform<P, SIGN, true, false>(w, A, B, TW, RT, t);   // padi layout throughout
        group_sync<P, true>();                       // the last stage has read A and B
        if (live) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int q = t + TA * e, k = q >> 1;
                if (OKS_IN(q, 2 * N, OKS_B_XCHG)) A[q] = w[e] * ((a.centred && (k & 1)) ? -sc_n2 : sc_n2);
            }
        }
        __syncthreads();
        // whole row segments out: chunk (r, j) is A_j[2r], A_j[2r + 1]
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * TC;
        float2* base = a.data + p * a.prob_stride + x0;
        for (int k = threadIdx.x; k < N * G; k += T * G) {
            const int r = k / G, j = k % G;
            if (x0 + 2 * j >= a.nx) continue;
            if (!OKS_IN(j * GS + 2 * r + 1, G * GS, OKS_B_STAGE)) continue;
            *reinterpret_cast<float4*>(base + (long long)r * a.nx + 2 * j) =
                *reinterpret_cast<const float4*>(AB + j * GS + 2 * r);
        }
    }
    cp_async_wait_all();
}

// ------------------------------------------------ columns across the lanes
// Column transform with the lanes running across CW adjacent columns: thread
// (c, tc) = (tid % CW, tid / CW) owns column x0 + c and the butterflies
// b = tc, tc + TPC, ... of every stage.  A half-warp (CW = 16) touches one
// row of 16 columns at a time, so stage 0 reads and the last stage writes
// whole 128-byte row segments straight from and to global memory, and the
// middle stages work in place on one [N][CW] shared-memory tile (each thread
// reads all its butterflies' inputs before the barrier that precedes the
// writes).  Twiddles depend on the row only: one broadcast per half-warp.
// PF: stage 0 reads its inputs from the staging tile ST ([N][CW], filled by
// cp.async while the previous tile was transformed) instead of global memory.
// Output pairs Q, Q + 1, ..., (R - 1) / 2 of a large odd-radix butterfly
// (symmetric form, compile-time roots) stored to the lanes tile.
template <int SIGN, int R, int Q, int CW>
__device__ __forceinline__ void lanes_odd_pairs(const float2* a, const float2* b, float2 x0, float2* D, int ob,
                                                int p, int c) {
    if constexpr (Q <= (R - 1) / 2) {
        float2 re = x0, im = make_float2(0.f, 0.f);
        odd_acc<R, Q, 1>(a, b, re, im);
        const float2 si = mul_si<SIGN>(im);
        D[(ob + Q * p) * CW + c] = re + si;
        D[(ob + (R - Q) * p) * CW + c] = re - si;
        lanes_odd_pairs<SIGN, R, Q + 1, CW>(a, b, x0, D, ob, p, c);
    }
}

// After every thread has read ST, refill() issues the next tile's copies.
struct NoRefill {
    __device__ void operator()() const {}
};
// Last-stage output: NoOut writes the column to global memory (centring
// sign and scale applied); any other functor receives (row, value).
struct NoOut {
    __device__ void operator()(int, float2) const {}
};
template <class P, int SIGN, int CW, int TPC, int s, bool PF = false, class F = NoRefill, class Out = NoOut>
__device__ __forceinline__ void lanes_stage(float2* __restrict__ D, const float2* __restrict__ TW,
                                            const float2* __restrict__ RT, float2* __restrict__ col, int nx,
                                            bool on, bool centred, float sc, int c, int tc,
                                            const float2* __restrict__ ST = nullptr, const F& refill = F(),
                                            const Out& out = Out()) {
    constexpr int S = P::S, N = P::N;
    constexpr int R = SIGN < 0 ? P::R[s] : P::R[S - 1 - s];
    constexpr int p = SIGN < 0 ? P::prod(s) : P::rprod(s);
    constexpr int off = SIGN < 0 ? Tw<P>::fwd(s) : Tw<P>::inv(s);
    constexpr int NB = N / R;
    constexpr int BPT = (NB + TPC - 1) / TPC;   // butterflies per thread
    if constexpr (R % 2 == 1 && R > 5) {
        // Large odd radix (the middle stage of 368 = 4·23·4): each thread folds
        // its butterflies' inputs, a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}
        // (twiddled), and after the barrier forms the output pairs with
        // compile-time roots; one thread per butterfly, no repeated folds.
        static_assert(s > 0 && s < S - 1, "the large odd radix is a middle stage");
        constexpr int H = (R - 1) / 2;
        float2 x0[BPT], fa[BPT][H], fb[BPT][H];
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB % TPC != 0 && b >= NB) break;
            const int k = b % p;
            x0[bb] = OKS_IN(b * CW + c, N * CW, OKS_B_TILE) ? D[b * CW + c] : make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                float2 u = D[(b + j * NB) * CW + c];
                float2 w = D[(b + (R - j) * NB) * CW + c];
                if (p > 1) {
                    u = twmul<SIGN>(u, TW[off + k * (R - 1) + j - 1]);
                    w = twmul<SIGN>(w, TW[off + k * (R - 1) + R - j - 1]);
                }
                fa[bb][j - 1] = u + w;
                fb[bb][j - 1] = u - w;
            }
        }
        __syncthreads();                                  // in place: all inputs read before any output lands
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB % TPC != 0 && b >= NB) break;
            const int k = b % p;
            const int ob = (b - k) * R + k;
            float2 y0 = x0[bb];
#pragma unroll
            for (int j = 0; j < H; ++j) y0 = y0 + fa[bb][j];
            if (OKS_IN((ob + (R - 1) * p) * CW + c, N * CW, OKS_B_TILE)) {
                D[ob * CW + c] = y0;
                lanes_odd_pairs<SIGN, R, 1, CW>(fa[bb], fb[bb], x0[bb], D, ob, p, c);
            }
        }
        __syncthreads();
        lanes_stage<P, SIGN, CW, TPC, s + 1, false, NoRefill, Out>(D, TW, RT, col, nx, on, centred, sc, c, tc, nullptr,
                                                                  NoRefill(), out);
        return;
    } else {
    float2 v[BPT][R];
#pragma unroll
    for (int bb = 0; bb < BPT; ++bb) {
        const int b = tc + TPC * bb;
        if (NB % TPC != 0 && b >= NB) break;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int r = b + j * NB;
            if constexpr (s == 0) {
                float2 x;
                if constexpr (PF) x = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
                else x = on ? col[r * nx] : make_float2(0.f, 0.f);   // N nx < 2^31 (launcher)
                if (centred && (r & 1)) x = make_float2(-x.x, -x.y);
                v[bb][j] = x;
            } else {
                v[bb][j] = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? D[r * CW + c] : make_float2(0.f, 0.f);
            }
        }
    }
    if constexpr (s > 0 && s < S - 1) __syncthreads();   // in place: all inputs read before any output lands
    if constexpr (PF && s == 0) {
        __syncthreads();                                  // ST read by every thread: refill it
        refill();
    }
#pragma unroll
    for (int bb = 0; bb < BPT; ++bb) {
        const int b = tc + TPC * bb;
        if (NB % TPC != 0 && b >= NB) break;
        const int k = b % p;
        if (p > 1) {
#pragma unroll
            for (int j = 1; j < R; ++j) v[bb][j] = twmul<SIGN>(v[bb][j], TW[off + k * (R - 1) + j - 1]);
        }
        bfly<SIGN, R>(v[bb], RT);
        const int ob = (b - k) * R + k;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int o = ob + j * p;
            if constexpr (s == S - 1) {
                if constexpr (std::is_same<Out, NoOut>::value) {
                    if (on) col[o * nx] = v[bb][j] * ((centred && (o & 1)) ? -sc : sc);
                } else {
                    out(o, v[bb][j]);
                }
            } else if (OKS_IN(o * CW + c, N * CW, OKS_B_TILE)) {
                D[o * CW + c] = v[bb][j];
            }
        }
    }
    if constexpr (s < S - 1) {
        __syncthreads();
        lanes_stage<P, SIGN, CW, TPC, s + 1, false, NoRefill, Out>(D, TW, RT, col, nx, on, centred, sc, c, tc, nullptr,
                                                                  NoRefill(), out);
    }
    }
}

// Register budget of the lanes form: 64, or 96 where a stage keeps more than
// 8 values per thread (radix 16, or two radix-8 butterflies).
template <class P, int TPC>
constexpr int lanes_regs() {
    int most = 0;
    for (int s = 0; s < P::S; ++s) {
        const int v = (P::N / P::R[s] + TPC - 1) / TPC * P::R[s];
        most = v > most ? v : most;
    }
    return most > 8 ? 96 : 64;
}

template <class P, int SIGN, int CW, int TPC, bool PF = false>
__global__ void __launch_bounds__(CW * TPC, xform_min_blocks<CW * TPC, lanes_regs<P, TPC>()>())
k_col_lanes(ColXformArgs a, const float2* __restrict__ gtw, const float2* __restrict__ groots, int roots_total) {
    constexpr int N = P::N;
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                  // [N][CW]
    float2* TWs = sm + N * CW;
    float2* RT = TWs + tw_half<P>();
    // PF: [N][CW] staging after the tables, on a 16-byte boundary
    float2* ST = sm + (((size_t)N * CW + tw_half<P>() + roots_total + 1) & ~size_t(1));
    const float2* TW = load_twiddles<P, SIGN>(TWs, gtw);
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    const int c = threadIdx.x % CW, tc = threadIdx.x / CW;
    const int ntx = (a.nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const float sc_n2 = (a.centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    if constexpr (PF) {
        // software-pipelined form: tile u + gridDim.x is copied into ST
        // (16-byte cp.async, whole row segments, L2 only) while tile u is
        // transformed; stage 0 reads ST.  nx is even and the rows start on
        // 16-byte boundaries (launcher), so chunks are whole.
        auto issue = [&](long long u) {
            const long long pr = u / ntx;
            const int x0 = (int)(u - pr * ntx) * CW;
            const float2* base = a.data + pr * a.prob_stride + x0;
            for (int k = threadIdx.x; k < N * (CW / 2); k += CW * TPC) {
                const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
                const bool on = x0 + j < a.nx;
                if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                    cp_async16(ST + r * CW + j, on ? base + (long long)r * a.nx + j : a.data, on ? 16u : 0u);
            }
            cp_async_commit();
        };
        long long u = blockIdx.x;
        if (u < total) issue(u);
        for (; u < total; u += gridDim.x) {
            const long long pr = u / ntx;
            const int x = (int)(u - pr * ntx) * CW + c;
            const bool on = x < a.nx;
            float2* col = a.data + pr * a.prob_stride + (on ? x : 0);
            cp_async_wait_all();
            __syncthreads();                         // ST holds tile u; the last tile's final stage has read D
            const long long un = u + gridDim.x;
            auto refill = [&]() {
                if (un < total) issue(un);
            };
            lanes_stage<P, SIGN, CW, TPC, 0, true>(D, TW, RT, col, (int)a.nx, on, a.centred != 0, sc_n2, c, tc, ST,
                                                   refill);
        }
        cp_async_wait_all();
        return;
    }
    for (long long u = blockIdx.x; u < total; u += gridDim.x) {
        const long long pr = u / ntx;
        const int x = (int)(u - pr * ntx) * CW + c;
        const bool on = x < a.nx;
        float2* col = a.data + pr * a.prob_stride + (on ? x : 0);
        __syncthreads();                             // tables loaded; the last tile's final stage has read D
        lanes_stage<P, SIGN, CW, TPC, 0>(D, TW, RT, col, (int)a.nx, on, a.centred != 0, sc_n2, c, tc);
    }
}

// Resident CTAs per SM of a kernel at a dynamic shared-memory size, queried
// once per (kernel, size) and device.
static int ctas_per_sm(const void* fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void*, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(fn, smem + ((size_t)dev << 40));
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess || n < 1) n = 1;
    cache[key] = n;
    return n;
}

static int sm_count() {
    static int n[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lk(mu);
    if (!n[dev]) cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev);
    return n[dev] > 0 ? n[dev] : 148;
}

template <class P>
static cudaError_t row_p(const RowXformArgs& a, cudaStream_t st) {
    constexpr int G = row_groups<P>();
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = cudaSuccess;
    if (a.tables) {   // caller-owned tables: nothing is allocated here
        tw = a.tables;
        rt = a.tables + Tw<P>::total();
        nrt = a.tables_nroots;
    } else if ((e = plan_tables<P>(&tw, &rt, &nrt)) != cudaSuccess) {
        return e;
    }
    const size_t smem = sizeof(float2) * ((size_t)G * 2 * (P::N + xbuf<P>()) + tw_half<P>() + nrt);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_row_xform_reg<P, -1>)
                                : reinterpret_cast<const void*>(k_row_xform_reg<P, +1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long units = (a.nrows + 1) / 2;
    long long grid = (units + G - 1) / G;
    const long long cap = (long long)ctas_per_sm(fn, P::T * G, smem) * sm_count();
    if (grid > cap) grid = cap;
    RowXformArgs b = a;
    b.vec16 = ((reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (a.ld_in & 1) == 0) ? 1 : 0;
    if (a.sign < 0) k_row_xform_reg<P, -1><<<(unsigned)grid, P::T * G, smem, st>>>(b, tw, rt, nrt);
    else k_row_xform_reg<P, +1><<<(unsigned)grid, P::T * G, smem, st>>>(b, tw, rt, nrt);
    return cudaGetLastError();
}

template <class P, int G>
static cudaError_t col_pg(const ColXformArgs& a, cudaStream_t st) {
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    const size_t smem =
        sizeof(float2) * ((size_t)P::N * (2 * G + 2) + (size_t)G * (2 * xbuf<P, false>() + 2) + tw_half<P>() + nrt);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_col_xform_reg<P, G, -1>)
                                : reinterpret_cast<const void*>(k_col_xform_reg<P, G, +1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + 2 * G - 1) / (2 * G));
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, P::T * G, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_col_xform_reg<P, G, -1><<<(unsigned)grid, P::T * G, smem, st>>>(a, tw, rt, nrt);
    else k_col_xform_reg<P, G, +1><<<(unsigned)grid, P::T * G, smem, st>>>(a, tw, rt, nrt);
    return cudaGetLastError();
}

template <class P, int CW, int TPC, bool PF>
static cudaError_t col_lanes_kp(const ColXformArgs& a, cudaStream_t st) {
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    size_t elems = (size_t)P::N * CW + tw_half<P>() + nrt;
    if (PF) elems = ((elems + 1) & ~size_t(1)) + (size_t)P::N * CW;
    const size_t smem = sizeof(float2) * elems;
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_col_lanes<P, -1, CW, TPC, PF>)
                                : reinterpret_cast<const void*>(k_col_lanes<P, +1, CW, TPC, PF>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + CW - 1) / CW);
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, CW * TPC, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_col_lanes<P, -1, CW, TPC, PF><<<(unsigned)grid, CW * TPC, smem, st>>>(a, tw, rt, nrt);
    else k_col_lanes<P, +1, CW, TPC, PF><<<(unsigned)grid, CW * TPC, smem, st>>>(a, tw, rt, nrt);
    return cudaGetLastError();
}

// The pipelined form needs whole 16-byte chunks: even nx, 16-byte aligned data.
template <class P, int CW, int TPC>
static cudaError_t col_lanes_k(const ColXformArgs& a, cudaStream_t st) {
    const bool pf_ok = (a.nx % 2) == 0 && (reinterpret_cast<uintptr_t>(a.data) & 15) == 0;
    if (a.lanes_pf > 0 && pf_ok) return col_lanes_kp<P, CW, TPC, true>(a, st);
    return col_lanes_kp<P, CW, TPC, false>(a, st);
}

// Lanes form per column length, from B200 measurements on 1 GiB of planes
// (GB/s of the column pass; pipelined lanes form at its best (width,
// threads) choice / direct lanes form / tiles): 192 5074 / 4346 / 3368 (form
// 4), 256 5065 / 4807 / 4535 (form 4), 320 4528 / 3514 / 3177 (form 1), 384
// 4581 / 3782 / 4063 (form 3), 512 4805 / 4154 / 4144 (form 1), 640 4078 /
// 2784 / 3689 (form 2), 368 4158 / 2750 / 2624 (form 8, (8, 32): 32 threads
// per column, the radix-23 stage on 16 of them, one butterfly each).  The
// tiles stay at 128 (5043 / 3907 against the direct lanes form).  At 368 and
// 640 the two-stage forms replace them: 368 = 16 · 23 (form 9) 5244, 640 =
// 20 · 32 (form 10) 4575, and at 320: 16 · 20 (form 11) 5690.
template <class P>
constexpr int lanes_default() {
    return (P::N == 192 || P::N == 256) ? 4
           : P::N == 320 ? 11
           : P::N == 512 ? 1
           : P::N == 384 ? 3
           : P::N == 640 ? 10
           : P::N == 368 ? 9
                         : 0;
}

// Columns across the lanes: tile width CW and threads per column TPC
// (lanes 1..4: (16, 32), (16, 64), (8, 64), (8, 32)).
static cudaError_t col_q368(const ColXformArgs& a, cudaStream_t st);   // the two-stage 368 form (below)
static cudaError_t col_q640(const ColXformArgs& a, cudaStream_t st);   // the two-stage 640 form (below)
static cudaError_t col_q320(const ColXformArgs& a, cudaStream_t st);   // the two-stage 320 form (below)

template <class P>
static cudaError_t col_lanes(const ColXformArgs& a, int lanes, cudaStream_t st) {
    if constexpr (big_odd_plan<P>()) {
        if (lanes == 9 && P::N == 368 && (a.nx % 2) == 0 && (reinterpret_cast<uintptr_t>(a.data) & 15) == 0)
            return col_q368(a, st);
        // 16 threads per column: one per radix-23 butterfly (368 / 23 = 16);
        // 32: half of them idle in that stage, fewer butterflies each in the others
        if (lanes == 6) return col_lanes_k<P, 8, 16>(a, st);
        if (lanes == 7) return col_lanes_k<P, 16, 32>(a, st);
        if (lanes == 8) return col_lanes_k<P, 8, 32>(a, st);
        return col_lanes_k<P, 16, 16>(a, st);
    } else {
        if (lanes == 10 && P::N == 640 && (a.nx % 2) == 0 && (reinterpret_cast<uintptr_t>(a.data) & 15) == 0)
            return col_q640(a, st);
        if (lanes == 11 && P::N == 320 && (a.nx % 2) == 0 && (reinterpret_cast<uintptr_t>(a.data) & 15) == 0)
            return col_q320(a, st);
        switch (lanes) {
            case 2: return col_lanes_k<P, 16, 64>(a, st);
            case 3: return col_lanes_k<P, 8, 64>(a, st);
            case 4: return col_lanes_k<P, 8, 32>(a, st);
            default: return col_lanes_k<P, 16, 32>(a, st);
        }
    }
}

// Column pairs per tile: 8 (128-byte row segments) where 8 groups fit one
// CTA (1024 threads, 64 registers each) and one SM's shared memory, else 4.
template <class P>
static cudaError_t col_p(const ColXformArgs& a, cudaStream_t st) {
    {
        // columns across the lanes (in-problem offsets in 32 bits) where that
        // form measured faster than the tiles: 192, 256, 320, 368, 384, 512,
        // 640; 368 takes the forms 5-8, the other lengths 1-4
        int lanes = a.lanes != 0 ? a.lanes : lanes_default<P>();
        if (lanes > 0) {
            if constexpr (big_odd_plan<P>()) lanes = lanes < 5 ? 5 : lanes;   // 5-9
            else lanes = (lanes > 4 && !(lanes == 10 && P::N == 640) && !(lanes == 11 && P::N == 320)) ? 1 : lanes;
        }
        if (a.tile == 0 && lanes > 0 && (long long)P::N * a.nx < (1ll << 31)) return col_lanes<P>(a, lanes, st);
    }
    constexpr bool g8 = P::N <= 512 && P::T * 8 <= 1024 && !big_odd_plan<P>();
    int g = a.tile > 0 ? a.tile : (g8 ? 8 : 4);
    if (g >= 8 && P::N > 512) g = 4;
    if (g >= 8) return col_pg<P, 8>(a, st);
    if (g >= 4) return col_pg<P, 4>(a, st);
    return col_pg<P, 2>(a, st);
}

// 2-D-mask engine, column pass in the lanes form: one CTA per tile of CW
// columns of one problem (tiles without a sampled column are skipped).  The
// S tile comes in whole row segments (16-byte cp.async) into ST; the forward
// transform runs in place in D with the lanes across the columns, and its
// last stage writes the data residual m' (F S - y') back into ST; the
// inverse transform reads ST and its last stage writes S.  Same arithmetic
// as k2d_col_reg (plain DFTs of the modulated state, y' signed by
// (-1)^(r + x) and scaled by ysc); mode 0 forms S = F^H (m' y').
template <class P, int CW, int TPC>
__global__ void __launch_bounds__(CW * TPC, xform_min_blocks<CW * TPC, lanes_regs<P, TPC>()>())
k2d_col_lanes(Fista2dArgs a, int mode, const float2* __restrict__ gtw, const float2* __restrict__ groots,
              int roots_total) {
    constexpr int N = P::N;
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                  // [N][CW] transform stages
    float2* ST = sm + N * CW;                        // [N][CW] S tile (the next one lands here early)
    float2* RS = ST + N * CW;                        // [N][CW] F S, then the residual
    float2* TWs = RS + N * CW;                       // both directions' twiddles
    float2* RT = TWs + Tw<P>::total();
    for (int q = threadIdx.x; q < Tw<P>::total(); q += blockDim.x) TWs[q] = gtw[q];
    for (int q = threadIdx.x; q < roots_total; q += blockDim.x) RT[q] = groots[q];
    const int c = threadIdx.x % CW, tc = threadIdx.x / CW;
    const int nx = a.nx;
    const int ntx = (nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const float minv = a.minv, ysc = a.ysc;
    // tiles with a sampled column (the same answer in every thread)
    auto has_sample = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
        for (int cc = 0; cc < CW; ++cc) {
            const int xx = x0 + cc;
            if (xx < nx && ((__ldg(cb + (xx >> 5)) >> (xx & 31)) & 1u)) return true;
        }
        return false;
    };
    auto next_tile = [&](long long u) {
        for (; u < total; u += gridDim.x)
            if (has_sample(u)) break;
        return u;
    };
    // the S tile of unit u into ST: whole row segments, 16-byte cp.async
    auto issue = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const float2* S = a.S + p * a.st_stride;
        for (int k = threadIdx.x; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool onj = x0 + j < nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, onj ? S + (long long)r * nx + x0 + j : S, onj ? 16u : 0u);
        }
        cp_async_commit();
    };
    long long u = next_tile(blockIdx.x);
    if (mode && u < total) issue(u);
    while (u < total) {
        const long long un = next_tile(u + gridDim.x);
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* cb = a.colbits + mi * a.col_wstride;
        const int x = x0 + c;
        const bool on = x < nx;
        const bool colon = on && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u);
        const uint32_t* rb = a.rowbits + mi * a.row_wstride;
        const uint8_t* mk = a.mask + mi * a.mask_stride;
        float2* S = a.S + p * a.st_stride;
        const float2* y = a.y + p * a.y_stride;
        auto sampled = [&](int r) {
            return colon && (a.separable ? ((__ldg(rb + (r >> 5)) >> (r & 31)) & 1u) != 0 : mk[(long long)r * nx + x] != 0);
        };
        auto yprime = [&](int r) { return y[(long long)r * nx + x] * (((r + x) & 1) ? -ysc : ysc); };
        if (mode) {
            cp_async_wait_all();
            __syncthreads();                         // ST holds this tile; the last tile's inverse is done with D, RS
            // once the forward's first stage has read ST, the next tile's S
            // copy goes into it, in flight during both transforms
            auto refill = [&]() {
                if (un < total) issue(un);
            };
            float2* RSc = RS + c;
            auto keep = [RSc](int o, float2 v) { RSc[o * CW] = v; };
            lanes_stage<P, -1, CW, TPC, 0, true, decltype(refill), decltype(keep)>(D, TWs, RT, nullptr, nx, on, false,
                                                                                  1.f, c, tc, ST, refill, keep);
            __syncthreads();
            // the residual m' (F S - y') in place, each thread on its own column's rows
            for (int r = tc; r < N; r += TPC)
                RS[r * CW + c] = sampled(r) ? (RS[r * CW + c] - yprime(r)) * minv : make_float2(0.f, 0.f);
        } else {
            __syncthreads();                         // tables loaded; the last tile's inverse has read RS and D
            for (int r = tc; r < N; r += TPC) RS[r * CW + c] = sampled(r) ? yprime(r) * minv : make_float2(0.f, 0.f);
        }
        __syncthreads();                             // the residual tile is complete
        float2* Sc = S + (on ? x : 0);
        auto store = [Sc, on, nx](int o, float2 v) {
            if (on) Sc[(long long)o * nx] = v;
        };
        lanes_stage<P, +1, CW, TPC, 0, true, NoRefill, decltype(store)>(D, TWs, RT, nullptr, nx, on, false, 1.f, c,
                                                                       tc, RS, NoRefill(), store);
        u = un;
    }
    cp_async_wait_all();
}

template <class P, int CW, int TPC>
static cudaError_t col2d_lanes_k(const Fista2dArgs& a, int mode, cudaStream_t st) {
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)3 * P::N * CW + Tw<P>::total() + nrt);
    const void* fn = reinterpret_cast<const void*>(k2d_col_lanes<P, CW, TPC>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + CW - 1) / CW);
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, CW * TPC, smem) * sm_count();
    if (grid > cap) grid = cap;
    k2d_col_lanes<P, CW, TPC><<<(unsigned)grid, CW * TPC, smem, st>>>(a, mode, tw, rt, nrt);
    return cudaGetLastError();
}

template <class P>
static cudaError_t col2d_lanes(const Fista2dArgs& a, int form, int mode, cudaStream_t st) {
    if constexpr (big_odd_plan<P>()) {
        if (form == 6) return col2d_lanes_k<P, 8, 16>(a, mode, st);
        if (form == 7) return col2d_lanes_k<P, 16, 32>(a, mode, st);
        if (form == 8) return col2d_lanes_k<P, 8, 32>(a, mode, st);
        return col2d_lanes_k<P, 16, 16>(a, mode, st);
    } else {
        switch (form) {
            case 2: return col2d_lanes_k<P, 16, 64>(a, mode, st);
            case 3: return col2d_lanes_k<P, 8, 64>(a, mode, st);
            case 4: return col2d_lanes_k<P, 8, 32>(a, mode, st);
            default: return col2d_lanes_k<P, 16, 32>(a, mode, st);
        }
    }
}


// 2-D-mask engine, column pass at ny = 368 for separable masks, pruned to
// the sampled rows (forms 9-12).  The plan is 368 = 4 · 23 · 4 (Stockham,
// the inverse in reversed order).  With need[i] = "one of the rows i,
// i + 92, i + 184, i + 276 is sampled" (i < 92):
//  - forward: output o = ob + 4 j of radix-23 butterfly b (k = b mod 4) is
//    read only by last-stage butterfly o mod 92 = k + 4 j, whose outputs are
//    exactly those four rows.  Output pairs (j, 23 - j) with need[k + 4 j]
//    and need[k + 92 - 4 j] both clear are not formed, and the last stage
//    skips the butterflies i with need[i] clear (their rows are unsampled:
//    the residual there is zero and is written by the inverse's first stage);
//  - inverse: the residual is zero off the sampled rows, so first-stage
//    butterfly i has only zero inputs when need[i] is clear (it writes
//    zeros), and input pair (j, 23 - j) of radix-23 butterfly b is zero when
//    need[b/4 + 4 j] and need[b/4 + 92 - 4 j] are clear: its fold and its
//    terms are left out (each would add an exact zero).
// Both tests depend on the butterfly only through its class (b mod 4
// forward, b / 4 inverse).  The forward maps thread tc < 16 to butterfly
// 4 (tc mod 4) + tc / 4 and the inverse to butterfly tc, so in both the
// class is tc / 4 and every warp's branches are uniform.  Tiles of CW
// columns with the lanes across the columns as in k2d_col_lanes; the S tile
// of the next unit is staged by 16-byte cp.async into ST once the forward's
// first stage has read it; D holds every stage in place.  Same arithmetic
// per formed output as the full transform.
// D row slot of row r in k2d_col_p368.  SW (form 13): rows r and r ^ 1 trade
// places when bit 2 of r is set, so the strided row sets of the stages fall on
// both halves of the banks (a permutation inside each row pair: the slots stay
// in [0, N)).  On B200 it removed 84 % of the shared-memory bank conflicts but
// added 16 % instructions; the forms 9-12 keep the rows in order.
template <bool SW>
__device__ __forceinline__ int p368_slot(int r) {
    if constexpr (SW) return r ^ ((r >> 2) & 1);
    else return r;
}

template <int CW, bool SW, int SIGN, int Q>
__device__ __forceinline__ void p368_pairs_fwd(const float2* fa, const float2* fb, float2 x0, float2* D, int ob,
                                               int c, uint32_t pm) {
    if constexpr (Q <= 11) {
        if ((pm >> Q) & 1u) {
            float2 re = x0, im = make_float2(0.f, 0.f);
            odd_acc<23, Q, 1>(fa, fb, re, im);
            const float2 si = mul_si<SIGN>(im);
            D[p368_slot<SW>(ob + 4 * Q) * CW + c] = re + si;
            D[p368_slot<SW>(ob + 4 * (23 - Q)) * CW + c] = re - si;
        }
        p368_pairs_fwd<CW, SW, SIGN, Q + 1>(fa, fb, x0, D, ob, c, pm);
    }
}
// re += sum a_j cos(2 pi j Q / 23), im += sum b_j sin(...), over the j with pm bit j
template <int Q, int J>
__device__ __forceinline__ void p368_acc_masked(const float2* a, const float2* b, float2& re, float2& im,
                                                uint32_t pm) {
    if constexpr (J <= 11) {
        if ((pm >> J) & 1u) {
            constexpr int M = (J * Q) % 23;
            re.x = fmaf(a[J - 1].x, RootRM<23, M>::c, re.x);
            re.y = fmaf(a[J - 1].y, RootRM<23, M>::c, re.y);
            im.x = fmaf(b[J - 1].x, RootRM<23, M>::s, im.x);
            im.y = fmaf(b[J - 1].y, RootRM<23, M>::s, im.y);
        }
        p368_acc_masked<Q, J + 1>(a, b, re, im, pm);
    }
}
template <int CW, bool SW, int SIGN, int Q>
__device__ __forceinline__ void p368_pairs_inv(const float2* fa, const float2* fb, float2 x0, float2* D, int ob,
                                               int c, uint32_t pm) {
    if constexpr (Q <= 11) {
        float2 re = x0, im = make_float2(0.f, 0.f);
        p368_acc_masked<Q, 1>(fa, fb, re, im, pm);
        const float2 si = mul_si<SIGN>(im);
        D[p368_slot<SW>(ob + 4 * Q) * CW + c] = re + si;
        D[p368_slot<SW>(ob + 4 * (23 - Q)) * CW + c] = re - si;
        p368_pairs_inv<CW, SW, SIGN, Q + 1>(fa, fb, x0, D, ob, c, pm);
    }
}

template <int CW, int TPC, bool SW>
__global__ void __launch_bounds__(CW * TPC, 512 / (CW * TPC) > 0 ? 512 / (CW * TPC) : 1)   // 128 registers
k2d_col_p368(Fista2dArgs a, const float2* __restrict__ gtw) {
    using P = S368;
    constexpr int N = 368, NB4 = 92, H = 11;
    constexpr int BPT = (NB4 + TPC - 1) / TPC;   // radix-4 butterflies per thread
    static_assert(TPC >= 16 && CW * TPC >= 108, "16 radix-23 butterflies; 3 warps build the need bits");
    static_assert(CW % 2 == 0, "16-byte copies of column pairs");
    constexpr int F1 = Tw<P>::fwd(1), F2 = Tw<P>::fwd(2), I1 = Tw<P>::inv(1), I2 = Tw<P>::inv(2);
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                           // [N][CW] every stage, in place (row slots swizzled)
    float2* ST = sm + N * CW;                                 // [N][CW] S tile, then y' on the sampled rows
    float2* TWs = ST + N * CW;                                // both directions' twiddles
    uint32_t* NEED = reinterpret_cast<uint32_t*>(TWs + Tw<P>::total());   // 3 words: need[0..92)
    uint32_t* ROWS = NEED + 4;                                // 12 words: the tile's sampled rows
    for (int q = threadIdx.x; q < Tw<P>::total(); q += blockDim.x) TWs[q] = gtw[q];
    pdl_wait();                                       // the previous pass's S is complete
    pdl_trigger();
    const int tid = threadIdx.x, c = tid % CW, tc = tid / CW, lane = tid & 31;
    const int cls = (tc >> 2) & 3;                            // this thread's radix-23 class (tc < 16)
    const int nx = a.nx;
    const int ntx = (nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const float minv = a.minv, ysc = a.ysc;
    auto dr = [](int r) { return p368_slot<SW>(r) * CW; };
    auto has_sample = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
        for (int cc = 0; cc < CW; ++cc) {
            const int xx = x0 + cc;
            if (xx < nx && ((__ldg(cb + (xx >> 5)) >> (xx & 31)) & 1u)) return true;
        }
        return false;
    };
    auto next_tile = [&](long long u) {
        for (; u < total; u += gridDim.x)
            if (has_sample(u)) break;
        return u;
    };
    // the S tile of unit u into ST: whole row segments, 16-byte cp.async
    auto issue_s = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const float2* S = a.S + p * a.st_stride;
        for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool onj = x0 + j < nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, onj ? S + (long long)r * nx + x0 + j : S, onj ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto need = [&](int i) { return (NEED[i >> 5] >> (i & 31)) & 1u; };
    auto rowbit = [&](int r) { return (ROWS[r >> 5] >> (r & 31)) & 1u; };
    long long u = next_tile(blockIdx.x);
    if (u < total) issue_s(u);
    while (u < total) {
        const long long un = next_tile(u + gridDim.x);
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* rb = a.rowbits + mi * a.row_wstride;
        const int x = x0 + c;
        const bool on = x < nx;
        const bool colon = on && ((__ldg(a.colbits + mi * a.col_wstride + (x >> 5)) >> (x & 31)) & 1u);
        cp_async_wait_all();
        __syncthreads();                                      // ST holds this tile; the last tile is done with D, NEED, ROWS
        if (tid < 96) {
            const int i = tid;
            auto rbit = [&](int r) { return (__ldg(rb + (r >> 5)) >> (r & 31)) & 1u; };
            const bool bit = i < NB4 && (rbit(i) | rbit(i + 92) | rbit(i + 184) | rbit(i + 276));
            const uint32_t w = __ballot_sync(0xffffffffu, bit);
            if (lane == 0) NEED[tid >> 5] = w;
        } else if (tid < 108) {
            ROWS[tid - 96] = __ldg(rb + (tid - 96));
        }
        // forward stage 0 (radix 4, p = 1): inputs b + 92 j from ST
        float2 v[BPT][4];
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB4 % TPC != 0 && b >= NB4) break;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = b + NB4 * j;
                v[bb][j] = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();                                      // ST read by every thread; NEED and ROWS complete
        // pair masks of this thread's class (bit 0: the DC input / output)
        uint32_t pm;
        {
            const int q = lane < 12 ? lane : 0;
            const bool bit = lane < 12 && (q == 0 ? need(cls) : (need(cls + 4 * q) | need(cls + 92 - 4 * q)));
            pm = __ballot_sync(0xffffffffu, bit);
        }
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB4 % TPC != 0 && b >= NB4) break;
            bfly4<-1>(v[bb]);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (OKS_IN(dr(4 * b + j) + c, N * CW, OKS_B_TILE)) D[dr(4 * b + j) + c] = v[bb][j];
        }
        {
            // y' on the sampled rows into ST (16-byte cp.async, column pairs),
            // in flight during the forward's radix-23 stage
            const float2* y = a.y + p * a.y_stride;
            for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
                const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
                if (!rowbit(r)) continue;
                const bool onj = x0 + j < nx;
                if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                    cp_async16(ST + r * CW + j, onj ? y + (long long)r * nx + x0 + j : y, onj ? 16u : 0u);
            }
            cp_async_commit();
        }
        __syncthreads();
        // forward stage 1 (radix 23, p = 4): butterfly 4 (tc mod 4) + tc / 4
        {
            float2 x0v = make_float2(0.f, 0.f), fa[H], fb[H];
            int ob = 0;
            const bool act = tc < 16;
            if (act) {
                const int b = 4 * (tc & 3) + (tc >> 2), k = b & 3;
                ob = (b - k) * 23 + k;
                x0v = D[dr(b) + c];
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    const float2 uu = twmul<-1>(D[dr(b + 16 * j) + c], TWs[F1 + k * 22 + j - 1]);
                    const float2 ww = twmul<-1>(D[dr(b + 16 * (23 - j)) + c], TWs[F1 + k * 22 + 22 - j]);
                    fa[j - 1] = uu + ww;
                    fb[j - 1] = uu - ww;
                }
            }
            __syncthreads();                                  // in place: every input read
            if (act && OKS_IN((ob + 88) * CW + c, N * CW, OKS_B_TILE)) {
                if (pm & 1u) {
                    float2 y0 = x0v;
#pragma unroll
                    for (int j = 0; j < H; ++j) y0 = y0 + fa[j];
                    D[dr(ob) + c] = y0;
                }
                p368_pairs_fwd<CW, SW, -1, 1>(fa, fb, x0v, D, ob, c, pm);
            }
        }
        cp_async_wait_all();                                  // this thread's y' copies
        __syncthreads();
        // forward stage 2 (radix 4, p = 92) and the residual m' (F S - y'),
        // each butterfly in place on its own four rows
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB4 % TPC != 0 && b >= NB4) break;
            if (!need(b)) continue;
            float2 w4[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = b + NB4 * j;
                float2 t = OKS_IN(dr(r) + c, N * CW, OKS_B_TILE) ? D[dr(r) + c] : make_float2(0.f, 0.f);
                if (j > 0) t = twmul<-1>(t, TWs[F2 + b * 3 + j - 1]);
                w4[j] = t;
            }
            bfly4<-1>(w4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = b + NB4 * j;
                const bool smp = colon && rowbit(r);
                const float2 yv = smp ? ST[r * CW + c] * (((r + x) & 1) ? -ysc : ysc) : make_float2(0.f, 0.f);
                if (OKS_IN(dr(r) + c, N * CW, OKS_B_TILE))
                    D[dr(r) + c] = smp ? (w4[j] - yv) * minv : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();                                      // ST (y') read by every thread
        if (un < total) issue_s(un);                          // the next S tile, in flight during the inverse
        // inverse stage 0 (radix 4, p = 1): inputs b + 92 j, outputs 4 b + j
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB4 % TPC != 0 && b >= NB4) break;
            const bool nz = need(b) != 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = b + NB4 * j;
                v[bb][j] = (nz && OKS_IN(dr(r) + c, N * CW, OKS_B_TILE)) ? D[dr(r) + c] : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();                                      // in place: every input read
#pragma unroll
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (NB4 % TPC != 0 && b >= NB4) break;
            if (need(b)) bfly4<+1>(v[bb]);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (OKS_IN(dr(4 * b + j) + c, N * CW, OKS_B_TILE)) D[dr(4 * b + j) + c] = v[bb][j];
        }
        __syncthreads();
        // inverse stage 1 (radix 23, p = 4): butterfly tc, zero input pairs left out
        {
            float2 x0v = make_float2(0.f, 0.f), fa[H], fb[H];
            int ob = 0;
            const bool act = tc < 16;
            if (act) {
                const int b = tc, k = b & 3;
                ob = (b - k) * 23 + k;
                x0v = D[dr(b) + c];
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    if ((pm >> j) & 1u) {
                        const float2 uu = twmul<+1>(D[dr(b + 16 * j) + c], TWs[I1 + k * 22 + j - 1]);
                        const float2 ww = twmul<+1>(D[dr(b + 16 * (23 - j)) + c], TWs[I1 + k * 22 + 22 - j]);
                        fa[j - 1] = uu + ww;
                        fb[j - 1] = uu - ww;
                    } else {
                        fa[j - 1] = make_float2(0.f, 0.f);
                        fb[j - 1] = make_float2(0.f, 0.f);
                    }
                }
            }
            __syncthreads();                                  // in place: every input read
            if (act && OKS_IN((ob + 88) * CW + c, N * CW, OKS_B_TILE)) {
                float2 y0 = x0v;
#pragma unroll
                for (int j = 1; j <= H; ++j)
                    if ((pm >> j) & 1u) y0 = y0 + fa[j - 1];
                D[dr(ob) + c] = y0;
                p368_pairs_inv<CW, SW, +1, 1>(fa, fb, x0v, D, ob, c, pm);
            }
        }
        __syncthreads();
        // inverse stage 2 (radix 4, p = 92): rows b + 92 j of S
        {
            float2* Sc = a.S + p * a.st_stride + (on ? x : 0);
#pragma unroll
            for (int bb = 0; bb < BPT; ++bb) {
                const int b = tc + TPC * bb;
                if (NB4 % TPC != 0 && b >= NB4) break;
                float2 w4[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int r = b + NB4 * j;
                    float2 t = OKS_IN(dr(r) + c, N * CW, OKS_B_TILE) ? D[dr(r) + c] : make_float2(0.f, 0.f);
                    if (j > 0) t = twmul<+1>(t, TWs[I2 + b * 3 + j - 1]);
                    w4[j] = t;
                }
                bfly4<+1>(w4);
                if (on) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) Sc[(long long)(b + NB4 * j) * nx] = w4[j];
                }
            }
        }
        u = un;
    }
    cp_async_wait_all();
}

template <int CW, int TPC, bool SW = false>
static cudaError_t col2d_p368_k(const Fista2dArgs& a, cudaStream_t st) {
    using P = S368;
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)2 * P::N * CW + Tw<P>::total()) + 16 * sizeof(uint32_t);
    const void* fn = reinterpret_cast<const void*>(k2d_col_p368<CW, TPC, SW>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + CW - 1) / CW);
    long long grid = tiles;
    int per = ctas_per_sm(fn, CW * TPC, smem);
    if (a.col_ctas > 0 && a.col_ctas < per) per = a.col_ctas;
    const long long cap = (long long)per * sm_count();
    if (grid > cap) grid = cap;
    return launch_pass(k2d_col_p368<CW, TPC, SW>, (unsigned)grid, CW * TPC, smem, st, a.pdl != 0, a, tw);
}

// 2-D-mask engine, column pass at ny = 368 in two stages, 16 · 23, pruned to
// the sampled rows with the residual fused between the two directions (form
// 14).  Forward: radix 16 (p = 1), then radix 23 (p = 16), whose butterfly b
// produces exactly rows b + 16 j; the inverse, in reversed order, starts with
// radix 23 (p = 1) reading the same rows b + 16 j.  So one thread per radix-23
// butterfly folds the forward's inputs, forms only the output pairs (j,
// 23 - j) with a sampled row, takes the residual m' (F S - y') on them in
// registers and folds it straight into the inverse's radix-23 butterfly,
// where the pairs whose rows are both unsampled are zero and left out; it
// writes the inverse's 23 outputs.  The last stage is the inverse radix 16
// (p = 23), stored to S.  y' is copied by each thread for its own rows and
// column (8-byte cp.async into the staging tile once the first stage has read
// it), so no barrier guards it.  The pair masks depend on the butterfly's
// rows; forward butterfly 4 (tc mod 4) + tc / 4 puts the four butterflies of
// one class b mod 4 in each warp, so for masks sampled every 2nd or 4th row
// the branches are nearly uniform per warp.
// Twiddles (gtw, forward sign): [16][22] w_368^(j b) of the forward radix-23
// stage, then [23][15] w_368^(j b) of the inverse radix-16 stage (conjugated).
// Forward output pairs Q.. of radix-23 butterfly (fa, fb, x0) with a sampled
// row, their residual, and the inverse's folds ra = r_Q + r_(23-Q),
// rb = r_Q - r_(23-Q) (zero for a pair left out).  res(row, v) is the residual.
template <int Q, class Res>
__device__ __forceinline__ void q368_fwd_pairs(const float2* fa, const float2* fb, float2 x0, int b, uint32_t pm,
                                               const Res& res, float2* ra, float2* rb) {
    if constexpr (Q <= 11) {
        if ((pm >> Q) & 1u) {
            float2 re = x0, im = make_float2(0.f, 0.f);
            odd_acc<23, Q, 1>(fa, fb, re, im);
            const float2 si = mul_si<-1>(im);
            const float2 r1 = res(b + 16 * Q, re + si), r2 = res(b + 16 * (23 - Q), re - si);
            ra[Q - 1] = r1 + r2;
            rb[Q - 1] = r1 - r2;
        } else {
            ra[Q - 1] = make_float2(0.f, 0.f);
            rb[Q - 1] = make_float2(0.f, 0.f);
        }
        q368_fwd_pairs<Q + 1>(fa, fb, x0, b, pm, res, ra, rb);
    }
}
// Inverse output pairs Q.. of radix-23 butterfly (ra, rb, r0), p = 1: outputs
// 23 b + Q and 23 b + 23 - Q of the tile D.
template <int CW, int Q>
__device__ __forceinline__ void q368_inv_pairs(const float2* ra, const float2* rb, float2 r0, float2* D, int b, int c,
                                               uint32_t pm) {
    if constexpr (Q <= 11) {
        float2 re = r0, im = make_float2(0.f, 0.f);
        p368_acc_masked<Q, 1>(ra, rb, re, im, pm);
        const float2 si = mul_si<+1>(im);
        D[(23 * b + Q) * CW + c] = re + si;
        D[(23 * b + 23 - Q) * CW + c] = re - si;
        q368_inv_pairs<CW, Q + 1>(ra, rb, r0, D, b, c, pm);
    }
}

template <int CW, int TPC>
__global__ void __launch_bounds__(CW * TPC, 512 / (CW * TPC) > 0 ? 512 / (CW * TPC) : 1)   // 128 registers
k2d_col_q368(Fista2dArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 368, NB16 = 23, H = 11;
    constexpr int BPT = (NB16 + TPC - 1) / TPC;   // radix-16 butterflies per thread
    constexpr int TWF = 16 * 22, TWN = TWF + 23 * 15;
    static_assert(TPC >= 16 && CW == 8, "16 radix-23 butterflies; four of one class per warp");
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                           // [N][CW] the stages, in place
    float2* ST = sm + N * CW;                                 // [N][CW] S tile, then y' on the sampled rows
    float2* TWs = ST + N * CW;
    uint32_t* ROWS = reinterpret_cast<uint32_t*>(TWs + TWN);  // 12 words: the tile's sampled rows
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    pdl_wait();                                               // the previous pass's S is complete
    pdl_trigger();
    const int tid = threadIdx.x, c = tid % CW, tc = tid / CW;
    const int nx = a.nx;
    const int ntx = (nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const float minv = a.minv, ysc = a.ysc;
    const bool act = tc < 16;                                 // owns a radix-23 butterfly
    const int b23 = 4 * (tc & 3) + ((tc >> 2) & 3);
    auto has_sample = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
        for (int cc = 0; cc < CW; ++cc) {
            const int xx = x0 + cc;
            if (xx < nx && ((__ldg(cb + (xx >> 5)) >> (xx & 31)) & 1u)) return true;
        }
        return false;
    };
    auto next_tile = [&](long long u) {
        for (; u < total; u += gridDim.x)
            if (has_sample(u)) break;
        return u;
    };
    auto issue_s = [&](long long u) {
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const float2* S = a.S + p * a.st_stride;
        for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool onj = x0 + j < nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, onj ? S + (long long)r * nx + x0 + j : S, onj ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto rowbit = [&](int r) { return (ROWS[r >> 5] >> (r & 31)) & 1u; };
    long long u = next_tile(blockIdx.x);
    if (u < total) issue_s(u);
    while (u < total) {
        const long long un = next_tile(u + gridDim.x);
        const long long p = u / ntx;
        const int x0 = (int)(u - p * ntx) * CW;
        const long long mi = (p + a.mask_offset) % a.mask_mod;
        const uint32_t* rb = a.rowbits + mi * a.row_wstride;
        const int x = x0 + c;
        const bool on = x < nx;
        const bool colon = on && ((__ldg(a.colbits + mi * a.col_wstride + (x >> 5)) >> (x & 31)) & 1u);
        cp_async_wait_all();
        __syncthreads();                                      // ST holds this tile; the last tile is done with D, ROWS
        if (tid < 12) ROWS[tid] = __ldg(rb + tid);
        // forward stage 0 (radix 16, p = 1): inputs b + 23 j from ST, outputs 16 b + j
#pragma unroll 1
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (b >= NB16) break;
            float2 v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int r = b + NB16 * j;
                v[j] = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
            }
            bfly16<-1>(v);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (OKS_IN((16 * b + j) * CW + c, N * CW, OKS_B_TILE)) D[(16 * b + j) * CW + c] = v[j];
        }
        __syncthreads();                                      // D complete; ST read by every thread; ROWS set
        // y' of this thread's own rows b23 + 16 j (sampled) and column into ST
        const float2* y = a.y + p * a.y_stride;
        if (act) {
#pragma unroll
            for (int j = 0; j < 23; ++j) {
                const int r = b23 + 16 * j;
                if (colon && rowbit(r) && OKS_IN(r * CW + c, N * CW, OKS_B_STAGE))
                    cp_async8(ST + r * CW + c, y + (long long)r * nx + x, 8u);
            }
        }
        cp_async_commit();
        // pair mask of this thread's butterfly: bit q set when row b23 + 16 q
        // or row b23 + 368 - 16 q is sampled (bit 0: row b23)
        uint32_t pm = 0;
        float2 x0v = make_float2(0.f, 0.f), fa[H], fb[H];
        if (act) {
            pm = rowbit(b23);
#pragma unroll
            for (int q = 1; q <= H; ++q) pm |= (rowbit(b23 + 16 * q) | rowbit(b23 + 368 - 16 * q)) << q;
            // forward radix-23 folds (p = 16: inputs b23 + 16 j, twiddles w^(j b23))
            x0v = D[b23 * CW + c];
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                const float2 uu = twmul<-1>(D[(b23 + 16 * j) * CW + c], TWs[b23 * 22 + j - 1]);
                const float2 ww = twmul<-1>(D[(b23 + 16 * (23 - j)) * CW + c], TWs[b23 * 22 + 22 - j]);
                fa[j - 1] = uu + ww;
                fb[j - 1] = uu - ww;
            }
        }
        __syncthreads();                                      // in place: every fold input read
        if (act) {
            cp_async_wait_all();                              // this thread's own y' copies
            auto res = [&](int r, float2 v) {
                const bool smp = colon && rowbit(r);
                return smp ? (v - ST[r * CW + c] * (((r + x) & 1) ? -ysc : ysc)) * minv : make_float2(0.f, 0.f);
            };
            float2 r0 = make_float2(0.f, 0.f);
            if (pm & 1u) {
                float2 y0 = x0v;
#pragma unroll
                for (int j = 0; j < H; ++j) y0 = y0 + fa[j];
                r0 = res(b23, y0);
            }
            float2 ra[H], rbv[H];
            q368_fwd_pairs<1>(fa, fb, x0v, b23, pm, res, ra, rbv);
            // inverse radix-23 (p = 1): outputs 23 b23 + j
            float2 y0 = r0;
#pragma unroll
            for (int j = 1; j <= H; ++j)
                if ((pm >> j) & 1u) y0 = y0 + ra[j - 1];
            if (OKS_IN((23 * b23 + 22) * CW + c, N * CW, OKS_B_TILE)) {
                D[(23 * b23) * CW + c] = y0;
                q368_inv_pairs<CW, 1>(ra, rbv, r0, D, b23, c, pm);
            }
        }
        __syncthreads();                                      // D complete; ST (y') read
        if (un < total) issue_s(un);                          // the next S tile, in flight during the last stage
        // inverse stage 1 (radix 16, p = 23): inputs b + 23 j, outputs rows b + 23 j of S
        float2* Sc = a.S + p * a.st_stride + (on ? x : 0);
#pragma unroll 1
        for (int bb = 0; bb < BPT; ++bb) {
            const int b = tc + TPC * bb;
            if (b >= NB16) break;
            float2 v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int r = b + NB16 * j;
                float2 t = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? D[r * CW + c] : make_float2(0.f, 0.f);
                if (j > 0) t = twmul<+1>(t, TWs[TWF + b * 15 + j - 1]);
                v[j] = t;
            }
            bfly16<+1>(v);
            if (on) {
#pragma unroll
                for (int j = 0; j < 16; ++j) Sc[(long long)(b + NB16 * j) * nx] = v[j];
            }
        }
        u = un;
    }
    cp_async_wait_all();
}

// Twiddles of k2d_col_q368 on the current device, built on first use.
static cudaError_t q368_tables(const float2** tw) {
    static float2* d_tab[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!d_tab[dev]) {
        const double two_pi = 6.283185307179586476925286766559;
        std::vector<float2> h;
        for (int b = 0; b < 16; ++b)
            for (int j = 1; j < 23; ++j) {
                const double ang = -two_pi * j * b / 368.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        for (int b = 0; b < 23; ++b)
            for (int j = 1; j < 16; ++j) {
                const double ang = -two_pi * j * b / 368.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        float2* d = nullptr;
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * h.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        d_tab[dev] = d;
    }
    *tw = d_tab[dev];
    return cudaSuccess;
}

static cudaError_t col2d_q368(const Fista2dArgs& a, cudaStream_t st) {
    constexpr int CW = 8, TPC = 16;
    const float2* tw;
    cudaError_t e = q368_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)2 * 368 * CW + 16 * 22 + 23 * 15) + 16 * sizeof(uint32_t);
    const void* fn = reinterpret_cast<const void*>(k2d_col_q368<CW, TPC>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + CW - 1) / CW);
    long long grid = tiles;
    int per = ctas_per_sm(fn, CW * TPC, smem);
    if (a.col_ctas > 0 && a.col_ctas < per) per = a.col_ctas;
    const long long cap = (long long)per * sm_count();
    if (grid > cap) grid = cap;
    return launch_pass(k2d_col_q368<CW, TPC>, (unsigned)grid, CW * TPC, smem, st, a.pdl != 0, a, tw);
}


// Standalone 368-point column transform in two stages, 16 · 23, with the
// lanes across 8 columns (xform_lanes 9).  Forward: radix 16 (p = 1) from the
// staging tile into D, then radix 23 (p = 16), one thread per butterfly,
// whose outputs are rows b + 16 j, stored straight to global memory (a warp
// writes four rows of 8 columns per step).  Inverse: radix 23 (p = 1) from
// the staging tile into D, then radix 16 (p = 23) storing rows b + 23 j.  One
// shared-memory exchange in either direction (the 4 · 23 · 4 form has two).
// Twiddles as k2d_col_q368.  Centring signs and scale as k_col_lanes.  The
// next tile's columns are copied into the staging tile (16-byte cp.async)
// once the first stage has read it: nx even and 16-byte aligned data.
template <int SIGN>
__device__ __forceinline__ void q368_out_pairs_store(const float2* fa, const float2* fb, float2 x0, float2* col,
                                                     int b, int nx, bool on, bool centred, float sc) {
    auto put = [&](int o, float2 v) {
        if (on) col[(long long)o * nx] = v * ((centred && (o & 1)) ? -sc : sc);
    };
    float2 y0 = x0;
#pragma unroll
    for (int j = 0; j < 11; ++j) y0 = y0 + fa[j];
    put(b, y0);
#define OKS_Q368_PAIR(Q)                                                   \
    {                                                                      \
        float2 re = x0, im = make_float2(0.f, 0.f);                        \
        odd_acc<23, Q, 1>(fa, fb, re, im);                                 \
        const float2 si = mul_si<SIGN>(im);                                \
        put(b + 16 * (Q), re + si);                                        \
        put(b + 16 * (23 - (Q)), re - si);                                 \
    }
    OKS_Q368_PAIR(1) OKS_Q368_PAIR(2) OKS_Q368_PAIR(3) OKS_Q368_PAIR(4) OKS_Q368_PAIR(5) OKS_Q368_PAIR(6)
    OKS_Q368_PAIR(7) OKS_Q368_PAIR(8) OKS_Q368_PAIR(9) OKS_Q368_PAIR(10) OKS_Q368_PAIR(11)
#undef OKS_Q368_PAIR
}

template <int SIGN>
__global__ void __launch_bounds__(128, 4)
k_col_q368(ColXformArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 368, CW = 8, TPC = 16, H = 11, TWF = 16 * 22, TWN = TWF + 23 * 15;
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                  // [N][CW]
    float2* ST = sm + N * CW;                        // [N][CW] staging
    float2* TWs = ST + N * CW;
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    const int tid = threadIdx.x, c = tid % CW, tc = tid / CW;
    const int ntx = (a.nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const bool centred = a.centred != 0;
    const float sc = (centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    auto issue = [&](long long u) {
        const long long pr = u / ntx;
        const int x0 = (int)(u - pr * ntx) * CW;
        const float2* base = a.data + pr * a.prob_stride + x0;
        for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool on = x0 + j < a.nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, on ? base + (long long)r * a.nx + j : a.data, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto ld = [&](int r) {                           // staged input, centring sign on load
        float2 x = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
        if (centred && (r & 1)) x = make_float2(-x.x, -x.y);
        return x;
    };
    long long u = blockIdx.x;
    if (u < total) issue(u);
    for (; u < total; u += gridDim.x) {
        const long long pr = u / ntx;
        const int x = (int)(u - pr * ntx) * CW + c;
        const bool on = x < a.nx;
        float2* col = a.data + pr * a.prob_stride + (on ? x : 0);
        const long long un = u + gridDim.x;
        cp_async_wait_all();
        __syncthreads();                             // ST holds tile u; the last tile is done with D
        if constexpr (SIGN < 0) {
            // radix 16 (p = 1): inputs b + 23 j, outputs 16 b + j
            float2 v[2][16];
#pragma unroll
            for (int bb = 0; bb < 2; ++bb) {
                const int b = tc + TPC * bb;
                if (b >= 23) break;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[bb][j] = ld(b + 23 * j);
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
#pragma unroll
            for (int bb = 0; bb < 2; ++bb) {
                const int b = tc + TPC * bb;
                if (b >= 23) break;
                bfly16<-1>(v[bb]);
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (OKS_IN((16 * b + j) * CW + c, N * CW, OKS_B_TILE)) D[(16 * b + j) * CW + c] = v[bb][j];
            }
            __syncthreads();
            // radix 23 (p = 16): butterfly tc, inputs tc + 16 j twiddled, outputs rows tc + 16 j
            if (tc < 16) {
                const int b = tc;
                float2 fa[H], fb[H];
                const float2 x0 = D[b * CW + c];
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    const float2 uu = twmul<-1>(D[(b + 16 * j) * CW + c], TWs[b * 22 + j - 1]);
                    const float2 ww = twmul<-1>(D[(b + 16 * (23 - j)) * CW + c], TWs[b * 22 + 22 - j]);
                    fa[j - 1] = uu + ww;
                    fb[j - 1] = uu - ww;
                }
                q368_out_pairs_store<-1>(fa, fb, x0, col, b, a.nx, on, centred, sc);
            }
        } else {
            // radix 23 (p = 1): butterfly tc, inputs tc + 16 j, outputs 23 tc + j
            float2 fa[H], fb[H], x0 = make_float2(0.f, 0.f);
            if (tc < 16) {
                x0 = ld(tc);
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    const float2 uu = ld(tc + 16 * j), ww = ld(tc + 16 * (23 - j));
                    fa[j - 1] = uu + ww;
                    fb[j - 1] = uu - ww;
                }
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
            if (tc < 16 && OKS_IN((23 * tc + 22) * CW + c, N * CW, OKS_B_TILE)) {
                float2 y0 = x0;
#pragma unroll
                for (int j = 0; j < H; ++j) y0 = y0 + fa[j];
                D[(23 * tc) * CW + c] = y0;
                q368_inv_pairs<CW, 1>(fa, fb, x0, D, tc, c, 0xFFFu);   // every pair
            }
            __syncthreads();
            // radix 16 (p = 23): inputs b + 23 j twiddled, outputs rows b + 23 j
#pragma unroll 1
            for (int bb = 0; bb < 2; ++bb) {
                const int b = tc + TPC * bb;
                if (b >= 23) break;
                float2 v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float2 t = D[(b + 23 * j) * CW + c];
                    if (j > 0) t = twmul<+1>(t, TWs[TWF + b * 15 + j - 1]);
                    v[j] = t;
                }
                bfly16<+1>(v);
                if (on) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int o = b + 23 * j;
                        col[(long long)o * a.nx] = v[j] * ((centred && (o & 1)) ? -sc : sc);
                    }
                }
            }
        }
    }
    cp_async_wait_all();
}

static cudaError_t col_q368(const ColXformArgs& a, cudaStream_t st) {
    const float2* tw;
    cudaError_t e = q368_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)2 * 368 * 8 + 16 * 22 + 23 * 15);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_col_q368<-1>)
                                : reinterpret_cast<const void*>(k_col_q368<+1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + 7) / 8);
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, 128, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_col_q368<-1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    else k_col_q368<+1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    return cudaGetLastError();
}


// Standalone 368-point row transform in two stages, 16 · 23, 8 rows per CTA
// (xform_row_variant 3).  The rows are staged row-major by 16-byte cp.async
// (rows on 16-byte boundaries) while the previous tile is transformed.
// Forward: radix 16 (p = 1), item (r, b), b < 23, reads elements b + 23 j of
// row r from the staging tile and writes 16 b + j to D, whose rows are padded
// (index k + k / 16) so the stride-16 writes spread over the banks; radix 23
// (p = 16), thread (r, b) with b < 16, reads b + 16 j and stores elements
// b + 16 j of the row to global memory (16 consecutive elements per
// half-warp).  Inverse: radix 23 (p = 1) from the staging tile into D at
// 23 b + j, then radix 16 (p = 23) storing elements b + 23 j.  Twiddles as
// k2d_col_q368; kept rows, rowsign, centring and scale as k_row_xform_reg.
__device__ __forceinline__ int q368_pad(int k) { return k + (k >> 4); }

template <int SIGN>
__global__ void __launch_bounds__(128, 4)
k_row_q368(RowXformArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 368, RW = 8, NP = N + N / 16, H = 11, TWF = 16 * 22, TWN = TWF + 23 * 15;
    extern __shared__ __align__(16) float2 sm[];
    float2* ST = sm;                                 // [RW][N] staged rows
    float2* D = ST + RW * N;                         // [RW][NP] the exchange, padded rows
    float2* TWs = D + RW * NP;
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    const int tid = threadIdx.x;
    const long long ntiles = (a.nrows + RW - 1) / RW;
    const bool centred = a.centred != 0;
    const float sc_n2 = (centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    auto row_kept = [&](long long row) {
        if (row >= a.nrows) return false;
        return !a.use_keep || row_on(a.keep, row / a.rows_per_prob, (int)(row % a.rows_per_prob));
    };
    auto issue = [&](long long u) {
        for (int k = tid; k < RW * (N / 2); k += 128) {
            const int r = k / (N / 2), x = 2 * (k - r * (N / 2));
            const long long row = u * RW + r;
            const bool on = row_kept(row);
            if (OKS_IN(r * N + x + 1, RW * N, OKS_B_STAGE))
                cp_async16(ST + r * N + x, on ? a.in + row * a.ld_in + x : a.in, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto ld = [&](int r, int e) {                    // staged element e of row r, centring sign on load
        float2 v = OKS_IN(r * N + e, RW * N, OKS_B_TILE) ? ST[r * N + e] : make_float2(0.f, 0.f);
        if (centred && (e & 1)) v = make_float2(-v.x, -v.y);
        return v;
    };
    auto dd = [&](int r, int k) -> float2& { return D[r * NP + q368_pad(k)]; };
    long long u = blockIdx.x;
    if (u < ntiles) issue(u);
    for (; u < ntiles; u += gridDim.x) {
        const long long un = u + gridDim.x;
        // the output row of the radix-23 / radix-16 items is set per item below
        auto store = [&](int r, int e, float2 v) {
            const long long row = u * RW + r;
            if (row >= a.nrows) return;
            float s = sc_n2;
            if (a.rowsign && ((row % a.rows_per_prob) & 1)) s = -s;
            a.out[row * a.ld_out + e] = v * ((centred && (e & 1)) ? -s : s);
        };
        cp_async_wait_all();
        __syncthreads();                             // ST holds tile u; the last tile is done with D
        if constexpr (SIGN < 0) {
            // radix 16 (p = 1): items f = tid, tid + 128 < 184: (r, b) = (f / 23, f % 23)
            float2 v[2][16];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * 23) break;
                const int r = f / 23, b = f - r * 23;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[k][j] = ld(r, b + 23 * j);
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < ntiles) issue(un);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * 23) break;
                const int r = f / 23, b = f - r * 23;
                bfly16<-1>(v[k]);
#pragma unroll
                for (int j = 0; j < 16; ++j) dd(r, 16 * b + j) = v[k][j];
            }
            __syncthreads();
            // radix 23 (p = 16): thread (r, b) = (tid / 16, tid % 16)
            {
                const int r = tid >> 4, b = tid & 15;
                float2 fa[H], fb[H];
                const float2 x0 = dd(r, b);
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    const float2 uu = twmul<-1>(dd(r, b + 16 * j), TWs[b * 22 + j - 1]);
                    const float2 ww = twmul<-1>(dd(r, b + 16 * (23 - j)), TWs[b * 22 + 22 - j]);
                    fa[j - 1] = uu + ww;
                    fb[j - 1] = uu - ww;
                }
                float2 y0 = x0;
#pragma unroll
                for (int j = 0; j < H; ++j) y0 = y0 + fa[j];
                store(r, b, y0);
#define OKS_RQ368_PAIR(Q)                                                   \
                {                                                           \
                    float2 re = x0, im = make_float2(0.f, 0.f);             \
                    odd_acc<23, Q, 1>(fa, fb, re, im);                      \
                    const float2 si = mul_si<-1>(im);                       \
                    store(r, b + 16 * (Q), re + si);                        \
                    store(r, b + 16 * (23 - (Q)), re - si);                 \
                }
                OKS_RQ368_PAIR(1) OKS_RQ368_PAIR(2) OKS_RQ368_PAIR(3) OKS_RQ368_PAIR(4) OKS_RQ368_PAIR(5)
                OKS_RQ368_PAIR(6) OKS_RQ368_PAIR(7) OKS_RQ368_PAIR(8) OKS_RQ368_PAIR(9) OKS_RQ368_PAIR(10)
                OKS_RQ368_PAIR(11)
#undef OKS_RQ368_PAIR
            }
        } else {
            // radix 23 (p = 1): thread (r, b) = (tid / 16, tid % 16), inputs b + 16 j
            const int r = tid >> 4, b = tid & 15;
            float2 fa[H], fb[H];
            const float2 x0 = ld(r, b);
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                const float2 uu = ld(r, b + 16 * j), ww = ld(r, b + 16 * (23 - j));
                fa[j - 1] = uu + ww;
                fb[j - 1] = uu - ww;
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < ntiles) issue(un);
            {
                float2 y0 = x0;
#pragma unroll
                for (int j = 0; j < H; ++j) y0 = y0 + fa[j];
                dd(r, 23 * b) = y0;
#define OKS_RQ368_IPAIR(Q)                                                  \
                {                                                           \
                    float2 re = x0, im = make_float2(0.f, 0.f);             \
                    odd_acc<23, Q, 1>(fa, fb, re, im);                      \
                    const float2 si = mul_si<+1>(im);                       \
                    dd(r, 23 * b + (Q)) = re + si;                          \
                    dd(r, 23 * b + 23 - (Q)) = re - si;                     \
                }
                OKS_RQ368_IPAIR(1) OKS_RQ368_IPAIR(2) OKS_RQ368_IPAIR(3) OKS_RQ368_IPAIR(4) OKS_RQ368_IPAIR(5)
                OKS_RQ368_IPAIR(6) OKS_RQ368_IPAIR(7) OKS_RQ368_IPAIR(8) OKS_RQ368_IPAIR(9) OKS_RQ368_IPAIR(10)
                OKS_RQ368_IPAIR(11)
#undef OKS_RQ368_IPAIR
            }
            __syncthreads();
            // radix 16 (p = 23): items f < 184: (r, b) = (f / 23, f % 23), elements b + 23 j
#pragma unroll 1
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * 23) break;
                const int rr = f / 23, bb = f - rr * 23;
                float2 v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float2 t = dd(rr, bb + 23 * j);
                    if (j > 0) t = twmul<+1>(t, TWs[TWF + bb * 15 + j - 1]);
                    v[j] = t;
                }
                bfly16<+1>(v);
#pragma unroll
                for (int j = 0; j < 16; ++j) store(rr, bb + 23 * j, v[j]);
            }
        }
    }
    cp_async_wait_all();
}

static cudaError_t row_q368(const RowXformArgs& a, cudaStream_t st) {
    const float2* tw;
    cudaError_t e = q368_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)8 * 368 + 8 * (368 + 23) + 16 * 22 + 23 * 15);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_row_q368<-1>)
                                : reinterpret_cast<const void*>(k_row_q368<+1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = (a.nrows + 7) / 8;
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, 128, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_row_q368<-1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    else k_row_q368<+1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    return cudaGetLastError();
}


// Radix-20 butterfly in registers, 20 = 4 · 5: a 4-point DFT over j1 of
// x[5 j1 + j2] for each j2, the twiddles w20^(j2 k1), a 5-point DFT over j2
// for each k1, output k1 + 4 k2 (w = e^(SIGN 2 pi i / 20); the twiddles are
// immediates).
template <int SIGN, int J2, int K1>
__device__ __forceinline__ float2 tw20(float2 a) {
    if constexpr (J2 == 0 || K1 == 0) return a;
    else return cmul(a, make_float2(RootRM<20, (J2 * K1) % 20>::c, SIGN * RootRM<20, (J2 * K1) % 20>::s));
}
template <int SIGN, int J2>
__device__ __forceinline__ void bfly20_cols(const float2* v, float2 (*A)[4]) {
    if constexpr (J2 < 5) {
        float2 t[4] = {v[J2], v[5 + J2], v[10 + J2], v[15 + J2]};
        bfly4<SIGN>(t);
        A[J2][0] = t[0];
        A[J2][1] = tw20<SIGN, J2, 1>(t[1]);
        A[J2][2] = tw20<SIGN, J2, 2>(t[2]);
        A[J2][3] = tw20<SIGN, J2, 3>(t[3]);
        bfly20_cols<SIGN, J2 + 1>(v, A);
    }
}
template <int SIGN>
__device__ __forceinline__ void bfly20(float2* v) {
    float2 A[5][4];
    bfly20_cols<SIGN, 0>(v, A);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 u[5] = {A[0][k1], A[1][k1], A[2][k1], A[3][k1], A[4][k1]};
        bfly5<SIGN>(u);
#pragma unroll
        for (int k2 = 0; k2 < 5; ++k2) v[k1 + 4 * k2] = u[k2];
    }
}

// Standalone 320-point row transform in two stages, 16 · 20, 8 rows per CTA
// (xform_row_variant 3, and the default at 320): the structure of k_row_q368
// with a radix-20 second stage (one butterfly of 20 points per thread, 16 per
// row).  Twiddles (forward sign): [16][19] w_320^(j b) of the forward radix-20
// stage, then [20][15] w_320^(j b) of the inverse radix-16 stage.
template <int SIGN>
__global__ void __launch_bounds__(128, 4)
k_row_q320(RowXformArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 320, RW = 8, NP = N + N / 16, NB16 = 20, TWF = 16 * 19, TWN = TWF + 20 * 15;
    extern __shared__ __align__(16) float2 sm[];
    float2* ST = sm;                                 // [RW][N] staged rows
    float2* D = ST + RW * N;                         // [RW][NP] the exchange, padded rows
    float2* TWs = D + RW * NP;
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    const int tid = threadIdx.x;
    const long long ntiles = (a.nrows + RW - 1) / RW;
    const bool centred = a.centred != 0;
    const float sc_n2 = (centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    auto row_kept = [&](long long row) {
        if (row >= a.nrows) return false;
        return !a.use_keep || row_on(a.keep, row / a.rows_per_prob, (int)(row % a.rows_per_prob));
    };
    auto issue = [&](long long u) {
        for (int k = tid; k < RW * (N / 2); k += 128) {
            const int r = k / (N / 2), x = 2 * (k - r * (N / 2));
            const long long row = u * RW + r;
            const bool on = row_kept(row);
            if (OKS_IN(r * N + x + 1, RW * N, OKS_B_STAGE))
                cp_async16(ST + r * N + x, on ? a.in + row * a.ld_in + x : a.in, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto ld = [&](int r, int e) {
        float2 v = OKS_IN(r * N + e, RW * N, OKS_B_TILE) ? ST[r * N + e] : make_float2(0.f, 0.f);
        if (centred && (e & 1)) v = make_float2(-v.x, -v.y);
        return v;
    };
    auto dd = [&](int r, int k) -> float2& { return D[r * NP + q368_pad(k)]; };
    long long u = blockIdx.x;
    if (u < ntiles) issue(u);
    for (; u < ntiles; u += gridDim.x) {
        const long long un = u + gridDim.x;
        auto store = [&](int r, int e, float2 v) {
            const long long row = u * RW + r;
            if (row >= a.nrows) return;
            float s = sc_n2;
            if (a.rowsign && ((row % a.rows_per_prob) & 1)) s = -s;
            a.out[row * a.ld_out + e] = v * ((centred && (e & 1)) ? -s : s);
        };
        cp_async_wait_all();
        __syncthreads();                             // ST holds tile u; the last tile is done with D
        const int r20 = tid >> 4, b20 = tid & 15;    // this thread's radix-20 butterfly
        if constexpr (SIGN < 0) {
            float2 v[2][16];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * NB16) break;
                const int r = f / NB16, b = f - r * NB16;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[k][j] = ld(r, b + NB16 * j);
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < ntiles) issue(un);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * NB16) break;
                const int r = f / NB16, b = f - r * NB16;
                bfly16<-1>(v[k]);
#pragma unroll
                for (int j = 0; j < 16; ++j) dd(r, 16 * b + j) = v[k][j];
            }
            __syncthreads();
            // radix 20 (p = 16): inputs b + 16 j twiddled, outputs b + 16 j
            float2 w[20];
#pragma unroll
            for (int j = 0; j < 20; ++j) {
                float2 t = dd(r20, b20 + 16 * j);
                if (j > 0) t = twmul<-1>(t, TWs[b20 * 19 + j - 1]);
                w[j] = t;
            }
            bfly20<-1>(w);
#pragma unroll
            for (int j = 0; j < 20; ++j) store(r20, b20 + 16 * j, w[j]);
        } else {
            // radix 20 (p = 1): inputs b + 16 j from ST, outputs 20 b + j
            float2 w[20];
#pragma unroll
            for (int j = 0; j < 20; ++j) w[j] = ld(r20, b20 + 16 * j);
            __syncthreads();                         // ST read by every thread: refill it
            if (un < ntiles) issue(un);
            bfly20<+1>(w);
#pragma unroll
            for (int j = 0; j < 20; ++j) dd(r20, 20 * b20 + j) = w[j];
            __syncthreads();
            // radix 16 (p = 20): inputs b + 20 j twiddled, outputs b + 20 j
#pragma unroll 1
            for (int k = 0; k < 2; ++k) {
                const int f = tid + 128 * k;
                if (f >= RW * NB16) break;
                const int rr = f / NB16, bb = f - rr * NB16;
                float2 v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float2 t = dd(rr, bb + NB16 * j);
                    if (j > 0) t = twmul<+1>(t, TWs[TWF + bb * 15 + j - 1]);
                    v[j] = t;
                }
                bfly16<+1>(v);
#pragma unroll
                for (int j = 0; j < 16; ++j) store(rr, bb + NB16 * j, v[j]);
            }
        }
    }
    cp_async_wait_all();
}

static cudaError_t q320_tables(const float2** tw) {
    static float2* d_tab[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!d_tab[dev]) {
        const double two_pi = 6.283185307179586476925286766559;
        std::vector<float2> h;
        for (int b = 0; b < 16; ++b)
            for (int j = 1; j < 20; ++j) {
                const double ang = -two_pi * j * b / 320.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        for (int b = 0; b < 20; ++b)
            for (int j = 1; j < 16; ++j) {
                const double ang = -two_pi * j * b / 320.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        float2* d = nullptr;
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * h.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        d_tab[dev] = d;
    }
    *tw = d_tab[dev];
    return cudaSuccess;
}

static cudaError_t row_q320(const RowXformArgs& a, cudaStream_t st) {
    const float2* tw;
    cudaError_t e = q320_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)8 * 320 + 8 * (320 + 20) + 16 * 19 + 20 * 15);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_row_q320<-1>)
                                : reinterpret_cast<const void*>(k_row_q320<+1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = (a.nrows + 7) / 8;
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, 128, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_row_q320<-1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    else k_row_q320<+1><<<(unsigned)grid, 128, smem, st>>>(a, tw);
    return cudaGetLastError();
}


// Radix-32 butterfly in registers: two 16-point DFTs of the even and the odd
// inputs, then X[k] = E[k] + w32^k O[k], X[k + 16] = E[k] - w32^k O[k]
// (immediate twiddles).
template <int SIGN, int K>
__device__ __forceinline__ void bfly32_join(const float2* e, const float2* o, float2* v) {
    if constexpr (K < 16) {
        const float2 t = K == 0 ? o[K] : cmul(o[K], make_float2(RootRM<32, K>::c, SIGN * RootRM<32, K>::s));
        v[K] = e[K] + t;
        v[K + 16] = e[K] - t;
        bfly32_join<SIGN, K + 1>(e, o, v);
    }
}
template <int SIGN>
__device__ __forceinline__ void bfly32(float2* v) {
    float2 e[16], o[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        e[k] = v[2 * k];
        o[k] = v[2 * k + 1];
    }
    bfly16<SIGN>(e);
    bfly16<SIGN>(o);
    bfly32_join<SIGN, 0>(e, o, v);
}

// Standalone 640-point column transform in two stages, 20 · 32, with the
// lanes across 8 columns and 32 threads per column (xform_lanes 10).
// Forward: radix 20 (p = 1), thread tc owns butterfly tc (inputs tc + 32 j,
// outputs 20 tc + j) from the staging tile into D; radix 32 (p = 20), threads
// tc < 20, inputs tc + 20 j twiddled w_640^(j tc), outputs rows tc + 20 j
// straight to global memory.  Inverse: radix 32 (p = 1) from the staging
// tile (outputs 32 b + j), then radix 20 (p = 32), outputs rows b + 32 j.
// Twiddles (forward sign): [20][31] w_640^(j b), then [32][19] w_640^(j b).
template <int SIGN>
__global__ void __launch_bounds__(256, 2)
k_col_q640(ColXformArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 640, CW = 8, TPC = 32, TWF = 20 * 31, TWN = TWF + 32 * 19;
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                  // [N][CW]
    float2* ST = sm + N * CW;                        // [N][CW] staging
    float2* TWs = ST + N * CW;
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    const int tid = threadIdx.x, c = tid % CW, tc = tid / CW;
    const int ntx = (a.nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const bool centred = a.centred != 0;
    const float sc = (centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    auto issue = [&](long long u) {
        const long long pr = u / ntx;
        const int x0 = (int)(u - pr * ntx) * CW;
        const float2* base = a.data + pr * a.prob_stride + x0;
        for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool on = x0 + j < a.nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, on ? base + (long long)r * a.nx + j : a.data, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto ld = [&](int r) {
        float2 x = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
        if (centred && (r & 1)) x = make_float2(-x.x, -x.y);
        return x;
    };
    long long u = blockIdx.x;
    if (u < total) issue(u);
    for (; u < total; u += gridDim.x) {
        const long long pr = u / ntx;
        const int x = (int)(u - pr * ntx) * CW + c;
        const bool on = x < a.nx;
        float2* col = a.data + pr * a.prob_stride + (on ? x : 0);
        const long long un = u + gridDim.x;
        auto put = [&](int o, float2 v) {
            if (on) col[(long long)o * a.nx] = v * ((centred && (o & 1)) ? -sc : sc);
        };
        cp_async_wait_all();
        __syncthreads();                             // ST holds tile u; the last tile is done with D
        if constexpr (SIGN < 0) {
            float2 w[20];
#pragma unroll
            for (int j = 0; j < 20; ++j) w[j] = ld(tc + 32 * j);
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
            bfly20<-1>(w);
#pragma unroll
            for (int j = 0; j < 20; ++j)
                if (OKS_IN((20 * tc + j) * CW + c, N * CW, OKS_B_TILE)) D[(20 * tc + j) * CW + c] = w[j];
            __syncthreads();
            if (tc < 20) {
                float2 v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float2 t = D[(tc + 20 * j) * CW + c];
                    if (j > 0) t = twmul<-1>(t, TWs[tc * 31 + j - 1]);
                    v[j] = t;
                }
                bfly32<-1>(v);
#pragma unroll
                for (int j = 0; j < 32; ++j) put(tc + 20 * j, v[j]);
            }
        } else {
            float2 v[32];
            if (tc < 20) {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = ld(tc + 20 * j);
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
            if (tc < 20) {
                bfly32<+1>(v);
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (OKS_IN((32 * tc + j) * CW + c, N * CW, OKS_B_TILE)) D[(32 * tc + j) * CW + c] = v[j];
            }
            __syncthreads();
            float2 w[20];
#pragma unroll
            for (int j = 0; j < 20; ++j) {
                float2 t = D[(tc + 32 * j) * CW + c];
                if (j > 0) t = twmul<+1>(t, TWs[TWF + tc * 19 + j - 1]);
                w[j] = t;
            }
            bfly20<+1>(w);
#pragma unroll
            for (int j = 0; j < 20; ++j) put(tc + 32 * j, w[j]);
        }
    }
    cp_async_wait_all();
}

static cudaError_t q640_tables(const float2** tw) {
    static float2* d_tab[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!d_tab[dev]) {
        const double two_pi = 6.283185307179586476925286766559;
        std::vector<float2> h;
        for (int b = 0; b < 20; ++b)
            for (int j = 1; j < 32; ++j) {
                const double ang = -two_pi * j * b / 640.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        for (int b = 0; b < 32; ++b)
            for (int j = 1; j < 20; ++j) {
                const double ang = -two_pi * j * b / 640.0;
                h.push_back(make_float2((float)cos(ang), (float)sin(ang)));
            }
        float2* d = nullptr;
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * h.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        d_tab[dev] = d;
    }
    *tw = d_tab[dev];
    return cudaSuccess;
}

static cudaError_t col_q640(const ColXformArgs& a, cudaStream_t st) {
    const float2* tw;
    cudaError_t e = q640_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)2 * 640 * 8 + 20 * 31 + 32 * 19);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_col_q640<-1>)
                                : reinterpret_cast<const void*>(k_col_q640<+1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + 7) / 8);
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, 256, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_col_q640<-1><<<(unsigned)grid, 256, smem, st>>>(a, tw);
    else k_col_q640<+1><<<(unsigned)grid, 256, smem, st>>>(a, tw);
    return cudaGetLastError();
}


// Standalone 320-point column transform in two stages, 16 · 20, with the
// lanes across 8 columns and 20 threads per column (xform_lanes 11).
// Forward: radix 16 (p = 1), thread tc owns butterfly tc (inputs tc + 20 j,
// outputs 16 tc + j); radix 20 (p = 16), threads tc < 16, inputs tc + 16 j
// twiddled w_320^(j tc), outputs rows tc + 16 j straight to global memory.
// Inverse: radix 20 (p = 1) on threads tc < 16 (outputs 20 tc + j), then
// radix 16 (p = 20), outputs rows tc + 20 j.  Twiddles as k_row_q320.
template <int SIGN>
__global__ void __launch_bounds__(160, 3)
k_col_q320(ColXformArgs a, const float2* __restrict__ gtw) {
    constexpr int N = 320, CW = 8, TPC = 20, TWF = 16 * 19, TWN = TWF + 20 * 15;
    extern __shared__ __align__(16) float2 sm[];
    float2* D = sm;                                  // [N][CW]
    float2* ST = sm + N * CW;                        // [N][CW] staging
    float2* TWs = ST + N * CW;
    for (int q = threadIdx.x; q < TWN; q += blockDim.x) TWs[q] = gtw[q];
    const int tid = threadIdx.x, c = tid % CW, tc = tid / CW;
    const int ntx = (a.nx + CW - 1) / CW;
    const long long total = a.nprob * ntx;
    const bool centred = a.centred != 0;
    const float sc = (centred && ((N / 2) & 1)) ? -a.scale : a.scale;
    auto issue = [&](long long u) {
        const long long pr = u / ntx;
        const int x0 = (int)(u - pr * ntx) * CW;
        const float2* base = a.data + pr * a.prob_stride + x0;
        for (int k = tid; k < N * (CW / 2); k += CW * TPC) {
            const int r = k / (CW / 2), j = 2 * (k % (CW / 2));
            const bool on = x0 + j < a.nx;
            if (OKS_IN(r * CW + j + 1, N * CW, OKS_B_STAGE))
                cp_async16(ST + r * CW + j, on ? base + (long long)r * a.nx + j : a.data, on ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto ld = [&](int r) {
        float2 x = OKS_IN(r * CW + c, N * CW, OKS_B_TILE) ? ST[r * CW + c] : make_float2(0.f, 0.f);
        if (centred && (r & 1)) x = make_float2(-x.x, -x.y);
        return x;
    };
    long long u = blockIdx.x;
    if (u < total) issue(u);
    for (; u < total; u += gridDim.x) {
        const long long pr = u / ntx;
        const int x = (int)(u - pr * ntx) * CW + c;
        const bool on = x < a.nx;
        float2* col = a.data + pr * a.prob_stride + (on ? x : 0);
        const long long un = u + gridDim.x;
        auto put = [&](int o, float2 v) {
            if (on) col[(long long)o * a.nx] = v * ((centred && (o & 1)) ? -sc : sc);
        };
        cp_async_wait_all();
        __syncthreads();                             // ST holds tile u; the last tile is done with D
        if constexpr (SIGN < 0) {
            float2 v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = ld(tc + 20 * j);
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
            bfly16<-1>(v);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (OKS_IN((16 * tc + j) * CW + c, N * CW, OKS_B_TILE)) D[(16 * tc + j) * CW + c] = v[j];
            __syncthreads();
            if (tc < 16) {
                float2 w[20];
#pragma unroll
                for (int j = 0; j < 20; ++j) {
                    float2 t = D[(tc + 16 * j) * CW + c];
                    if (j > 0) t = twmul<-1>(t, TWs[tc * 19 + j - 1]);
                    w[j] = t;
                }
                bfly20<-1>(w);
#pragma unroll
                for (int j = 0; j < 20; ++j) put(tc + 16 * j, w[j]);
            }
        } else {
            float2 w[20];
            if (tc < 16) {
#pragma unroll
                for (int j = 0; j < 20; ++j) w[j] = ld(tc + 16 * j);
            }
            __syncthreads();                         // ST read by every thread: refill it
            if (un < total) issue(un);
            if (tc < 16) {
                bfly20<+1>(w);
#pragma unroll
                for (int j = 0; j < 20; ++j)
                    if (OKS_IN((20 * tc + j) * CW + c, N * CW, OKS_B_TILE)) D[(20 * tc + j) * CW + c] = w[j];
            }
            __syncthreads();
            float2 v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float2 t = D[(tc + 20 * j) * CW + c];
                if (j > 0) t = twmul<+1>(t, TWs[TWF + tc * 15 + j - 1]);
                v[j] = t;
            }
            bfly16<+1>(v);
#pragma unroll
            for (int j = 0; j < 16; ++j) put(tc + 20 * j, v[j]);
        }
    }
    cp_async_wait_all();
}

static cudaError_t col_q320(const ColXformArgs& a, cudaStream_t st) {
    const float2* tw;
    cudaError_t e = q320_tables(&tw);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(float2) * ((size_t)2 * 320 * 8 + 16 * 19 + 20 * 15);
    const void* fn = a.sign < 0 ? reinterpret_cast<const void*>(k_col_q320<-1>)
                                : reinterpret_cast<const void*>(k_col_q320<+1>);
    if ((e = set_smem_attr(fn, smem)) != cudaSuccess) return e;
    const long long tiles = a.nprob * ((a.nx + 7) / 8);
    long long grid = tiles;
    const long long cap = (long long)ctas_per_sm(fn, 160, smem) * sm_count();
    if (grid > cap) grid = cap;
    if (a.sign < 0) k_col_q320<-1><<<(unsigned)grid, 160, smem, st>>>(a, tw);
    else k_col_q320<+1><<<(unsigned)grid, 160, smem, st>>>(a, tw);
    return cudaGetLastError();
}

}  // namespace reg

cudaError_t launch_fista2d_col_lanes(const Fista2dArgs& a, int form, int mode, cudaStream_t st) {
    if (a.nprob <= 0) return cudaSuccess;
    if (a.nx % 2 || (reinterpret_cast<uintptr_t>(a.S) & 15)) return cudaErrorInvalidValue;
    if (form >= 9) {
        // the pruned 368 forms: separable masks, the iteration pass (mode 1)
        if (a.ny != 368 || !a.separable || mode != 1) return cudaErrorInvalidValue;
        switch (form) {
            case 10: return reg::col2d_p368_k<8, 32>(a, st);
            case 11: return reg::col2d_p368_k<16, 16>(a, st);
            case 12: return reg::col2d_p368_k<16, 32>(a, st);
            case 13: return reg::col2d_p368_k<8, 16, true>(a, st);
            case 14: return reg::col2d_q368(a, st);
            default: return reg::col2d_p368_k<8, 16>(a, st);
        }
    }
    switch (a.ny) {
        case 128: return reg::col2d_lanes<reg::S128>(a, form, mode, st);
        case 192: return reg::col2d_lanes<reg::S192>(a, form, mode, st);
        case 256: return reg::col2d_lanes<reg::S256>(a, form, mode, st);
        case 320: return reg::col2d_lanes<reg::S320>(a, form, mode, st);
        case 368: return reg::col2d_lanes<reg::S368>(a, form, mode, st);
        case 384: return reg::col2d_lanes<reg::S384>(a, form, mode, st);
        case 512: return reg::col2d_lanes<reg::S512>(a, form, mode, st);
        case 640: return reg::col2d_lanes<reg::P640>(a, form, mode, st);
        default: return cudaErrorInvalidValue;
    }
}

bool xform_reg_supported(int n) {
    switch (n) {
        case 128: case 192: case 256: case 320: case 368: case 384: case 512: case 640: return true;
        default: return false;
    }
}

namespace reg {
// Row plans for 192 measured on B200 (GB/s of the row pass, 1 GiB of
// planes): 12·4·4 on 32 threads, four row pairs per CTA (P192), 5610; 4·12·4
// on 96 threads (R192), 4445; 8·3·8 on 48 of 64 threads (S192), 3864.  P192
// is the default.  Measured and not taken elsewhere: 640 = 4·4·10·4 (3.84
// against 4.73 TB/s), 320 = 4·5·4·4 (4.14 against 4.40) and 8·5·8 on 80 of 96
// threads (3.97 against 4.04), 368 on 184 threads (2.91 against 2.93).
using R192 = Plan<192, 96, 4, 12, 4>;
}  // namespace reg

cudaError_t launch_row_xform_reg(const RowXformArgs& a, int n, cudaStream_t st) {
    if (a.nrows <= 0) return cudaSuccess;
    // alternative row plans (option xform_row_variant), for measurement
    if (a.variant == 1 && !a.tables) {
        if (n == 192) return reg::row_p<reg::S192>(a, st);    // 8·3·8 on 48 of 64 threads
        if (n == 320) return reg::row_p<reg::V320>(a, st);    // 8·5·8 on 80 of 96 threads
    }
    if (a.variant == 2 && !a.tables && n == 192) return reg::row_p<reg::R192>(a, st);   // 4·12·4 on 96 threads
    // the two-stage 368 form (the default at 368: 3.94 against 3.36 TB/s on
    // B200): rows on 16-byte boundaries, library-owned tables
    if ((a.variant == 3 || a.variant == 0) && !a.tables && n == 368 &&
        (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (a.ld_in & 1) == 0)
        return reg::row_q368(a, st);
    // the two-stage 320 form (16 · 20; the default at 320: 5.53 against
    // 4.05 TB/s on B200)
    if ((a.variant == 3 || a.variant == 0) && !a.tables && n == 320 &&
        (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (a.ld_in & 1) == 0)
        return reg::row_q320(a, st);
    switch (n) {
        case 128: return reg::row_p<reg::S128>(a, st);
        case 192: return reg::row_p<reg::P192>(a, st);
        case 256: return reg::row_p<reg::S256>(a, st);
        case 320: return reg::row_p<reg::S320>(a, st);
        case 368: return reg::row_p<reg::S368>(a, st);
        case 384: return reg::row_p<reg::S384>(a, st);
        case 512: return reg::row_p<reg::S512>(a, st);
        case 640: return reg::row_p<reg::P640>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

namespace reg {
template <class P>
static int row_tables_p(float2* h, int cap, int* nroots) {
    if (cap < Tw<P>::total() + P::N) return 0;   // roots: at most one per radix point
    return host_plan_tables<P>(h, nroots);
}
}  // namespace reg

// The plans here must be the ones launch_row_xform_reg picks per length.
int row_xform_reg_tables(int n, float2* h, int cap, int* nroots) {
    switch (n) {
        case 128: return reg::row_tables_p<reg::S128>(h, cap, nroots);
        case 192: return reg::row_tables_p<reg::P192>(h, cap, nroots);
        case 256: return reg::row_tables_p<reg::S256>(h, cap, nroots);
        case 320: return reg::row_tables_p<reg::S320>(h, cap, nroots);
        case 368: return reg::row_tables_p<reg::S368>(h, cap, nroots);
        case 384: return reg::row_tables_p<reg::S384>(h, cap, nroots);
        case 512: return reg::row_tables_p<reg::S512>(h, cap, nroots);
        case 640: return reg::row_tables_p<reg::P640>(h, cap, nroots);
        default: return 0;
    }
}

cudaError_t launch_col_xform_reg(const ColXformArgs& a, cudaStream_t st) {
    if (a.nprob <= 0 || a.nx <= 0) return cudaSuccess;
    switch (a.ny) {
        case 128: return reg::col_p<reg::S128>(a, st);
        case 192: return reg::col_p<reg::S192>(a, st);
        case 256: return reg::col_p<reg::S256>(a, st);
        case 320: return reg::col_p<reg::S320>(a, st);
        case 368: return reg::col_p<reg::S368>(a, st);
        case 384: return reg::col_p<reg::S384>(a, st);
        case 512: return reg::col_p<reg::S512>(a, st);
        case 640: return reg::col_p<reg::P640>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace oks
