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
//     registers (R | E); intermediate stages exchange through padded shared
//     memory (index + index/32 keeps the strided writes conflict-free);
//   * the last forward stage, the data residual and the first inverse stage
//     (same radix) run back to back in registers;
//   * the 2x2 Haar blocks pair q^1 (column) and q^2 (row): two xor-shuffle
//     Hadamard steps forward, two back.
// Only y' in and the coil image out touch global memory.
#include <cuda_runtime.h>

#include "fft_dev.cuh"
#include "kernels.h"

namespace oks {
namespace reg {

// Exchange-buffer index: an XOR swizzle inside each aligned block of 16
// float2 (one 128-byte row of banks).  The Stockham writes stride by 2R
// elements across lanes; folding bits 3.. and 6.. of the index into the low
// four bits spreads those strides over all 16 8-byte bank slots.  A bank model
// of every stage of every plan gives 1.00-1.31x the conflict-free wavefront
// count (the former "+1 float2 per 32" padding: 1.25-1.75x).
__device__ __forceinline__ int padi(int i) { return i ^ (((i >> 3) ^ (i >> 6)) & 15); }

// 8-byte asynchronous global -> shared copy; src_bytes 0 writes zeros (the
// source address is then not read but must still be a valid pointer).
__device__ __forceinline__ void cp_async8(float2* dst, const float2* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int SIGN, int R>
__device__ __forceinline__ void bfly(float2* v, const float2* __restrict__ roots) {
    if constexpr (R == 2) bfly2<SIGN>(v);
    else if constexpr (R == 3) bfly3<SIGN>(v);
    else if constexpr (R == 4) bfly4<SIGN>(v);
    else if constexpr (R == 5) bfly5<SIGN>(v);
    else if constexpr (R == 8) bfly8<SIGN>(v);
    else if constexpr (R == 16) bfly16<SIGN>(v);
    else if constexpr (R == 6) {           // 3 x 2
        float2 a[3] = {v[0], v[2], v[4]}, b[3] = {v[1], v[3], v[5]};
        bfly3<SIGN>(a);
        bfly3<SIGN>(b);
        // w6^k = cos(pi k/3) + SIGN i sin(pi k/3)
        const float h = 0.86602540378443864676f;
        float2 b1 = cmul(b[1], make_float2(0.5f, SIGN * h));
        float2 b2 = cmul(b[2], make_float2(-0.5f, SIGN * h));
        v[0] = a[0] + b[0]; v[3] = a[0] - b[0];
        v[1] = a[1] + b1;   v[4] = a[1] - b1;
        v[2] = a[2] + b2;   v[5] = a[2] - b2;
    } else if constexpr (R == 10) {        // 5 x 2
        float2 a[5] = {v[0], v[2], v[4], v[6], v[8]}, b[5] = {v[1], v[3], v[5], v[7], v[9]};
        bfly5<SIGN>(a);
        bfly5<SIGN>(b);
        // w10^k = cos(pi k/5) + SIGN i sin(pi k/5)
        const float c1 = 0.80901699437494742410f, s1 = 0.58778525229247312917f;
        const float c2 = 0.30901699437494742410f, s2 = 0.95105651629515357212f;
        const float2 w[5] = {make_float2(1.f, 0.f), make_float2(c1, SIGN * s1), make_float2(c2, SIGN * s2),
                             make_float2(-c2, SIGN * s2), make_float2(-c1, SIGN * s1)};
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const float2 tb = cmul(b[k], w[k]);
            v[k] = a[k] + tb;
            v[k + 5] = a[k] - tb;
        }
    } else if constexpr (R == 12) {        // 3 x 4
        float2 a[4] = {v[0], v[3], v[6], v[9]}, b[4] = {v[1], v[4], v[7], v[10]}, c[4] = {v[2], v[5], v[8], v[11]};
        bfly4<SIGN>(a);
        bfly4<SIGN>(b);
        bfly4<SIGN>(c);
        // y[k + 4m] = sum_l w12^{l k} (DFT4 of x[l + 3n])[k] w3^{l m}
        const float c1 = 0.86602540378443864676f, s1 = 0.5f;
        const float2 w1[4] = {make_float2(1.f, 0.f), make_float2(c1, SIGN * s1), make_float2(s1, SIGN * c1),
                              make_float2(0.f, SIGN * 1.f)};
        const float2 w2[4] = {make_float2(1.f, 0.f), make_float2(s1, SIGN * c1), make_float2(-s1, SIGN * c1),
                              make_float2(-1.f, 0.f)};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float2 t[3] = {a[k], cmul(b[k], w1[k]), cmul(c[k], w2[k])};
            bfly3<SIGN>(t);
            v[k] = t[0]; v[k + 4] = t[1]; v[k + 8] = t[2];
        }
    } else {
        static_assert(R % 2 == 1, "unsupported even radix");
        bfly_odd<SIGN, R>(v, roots);
    }
}

// Plans: N, active threads TA, stage radices.
template <int N_, int TA_, int... Rs>
struct Plan {
    static constexpr int N = N_;
    static constexpr int TA = TA_;
    static constexpr int T = (TA_ + 31) / 32 * 32;
    static constexpr int E = 2 * N_ / TA_;
    static constexpr int S = sizeof...(Rs);
    static constexpr int R[S] = {Rs...};
    static_assert(2 * N_ % TA_ == 0, "TA must divide 2N");
    static_assert(TA_ % 4 == 0, "TA must be a multiple of 4");
    static constexpr int prod(int k) {   // product of the first k radices
        int p = 1;
        for (int s = 0; s < k; ++s) p *= R[s];
        return p;
    }
    static constexpr int rprod(int k) {  // product of the first k radices of the reversed order
        int p = 1;
        for (int s = 0; s < k; ++s) p *= R[S - 1 - s];
        return p;
    }
    static_assert(prod(S) == N_, "radices must multiply to N");
    static_assert(E % R[0] == 0 && E % R[S - 1] == 0, "first and last radix must divide E");
    static constexpr int SMEM_X = 2 * N_ + (2 * N_) / 32 + 1;   // padded exchange buffer (float2)
};

// Twiddle table offsets: forward stage s at tw_f(s), inverse stage s at
// tw_i(s); entries k*(R-1) + j-1 = w_{pR}^{jk} (forward sign).
template <class P>
struct Tw {
    static constexpr int fwd(int s) {
        int o = 0;
        for (int u = 0; u < s; ++u) o += P::prod(u) * (P::R[u] - 1);
        return o;
    }
    static constexpr int inv(int s) {
        int o = fwd(P::S);
        for (int u = 0; u < s; ++u) o += P::rprod(u) * (P::R[P::S - 1 - u] - 1);
        return o;
    }
    static constexpr int total() { return inv(P::S); }
};

// cos and sin of 2 pi m / R for compile-time m and R (Taylor series of the
// angle reduced to [-pi, pi], 30 terms: below double rounding there), so the
// odd-radix butterflies below multiply by immediates instead of loading a
// table of roots.
constexpr double cx_sin(double x) {
    double term = x, sum = x;
    for (int n = 1; n < 30; ++n) {
        term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double cx_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int n = 1; n < 30; ++n) {
        term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
        sum += term;
    }
    return sum;
}
template <int R, int M>
struct RootRM {
    static constexpr double ang = 6.283185307179586476925286766559 * (double)(2 * M <= R ? M : M - R) / (double)R;
    static constexpr float c = (float)cx_cos(ang);
    static constexpr float s = (float)cx_sin(ang);
};

// re += sum_j a_j cos(2 pi j Q / R), im += sum_j b_j sin(2 pi j Q / R), j = J..H
template <int R, int Q, int J>
__device__ __forceinline__ void odd_acc(const float2* a, const float2* b, float2& re, float2& im) {
    if constexpr (J <= (R - 1) / 2) {
        constexpr int M = (J * Q) % R;
        re.x = fmaf(a[J - 1].x, RootRM<R, M>::c, re.x);
        re.y = fmaf(a[J - 1].y, RootRM<R, M>::c, re.y);
        im.x = fmaf(b[J - 1].x, RootRM<R, M>::s, im.x);
        im.y = fmaf(b[J - 1].y, RootRM<R, M>::s, im.y);
        odd_acc<R, Q, J + 1>(a, b, re, im);
    }
}

// Output pairs Q, Q + NS, ... of an odd-radix butterfly in symmetric form.
template <int SIGN, int R, int NS, int Q>
__device__ __forceinline__ void odd_pairs(const float2* a, const float2* b, float2 x0, float2* dst, int ob, int p,
                                          int c) {
    if constexpr (Q <= (R - 1) / 2) {
        float2 re = x0, im = make_float2(0.f, 0.f);
        odd_acc<R, Q, 1>(a, b, re, im);
        const float2 si = mul_si<SIGN>(im);
        dst[padi(2 * (ob + Q * p) + c)] = re + si;
        dst[padi(2 * (ob + (R - Q) * p) + c)] = re - si;
        odd_pairs<SIGN, R, NS, Q + NS>(a, b, x0, dst, ob, p, c);
    }
}

// Thread s of a butterfly's NS threads forms the pairs q = s+1, s+1+NS, ...
template <int SIGN, int R, int NS, int S0>
__device__ __forceinline__ void odd_pairs_for(int s, const float2* a, const float2* b, float2 x0, float2* dst, int ob,
                                              int p, int c) {
    if constexpr (S0 < NS) {
        if (s == S0) odd_pairs<SIGN, R, NS, S0 + 1>(a, b, x0, dst, ob, p, c);
        else odd_pairs_for<SIGN, R, NS, S0 + 1>(s, a, b, x0, dst, ob, p, c);
    }
}

// One stage over smem for intermediate stages: items f = t + TA*b, both
// columns, any radix.  src/dst are padded exchange buffers.
template <class P, int SIGN, int R, int p>
__device__ __forceinline__ void stage_smem(const float2* __restrict__ src, float2* __restrict__ dst,
                                           const float2* __restrict__ tw, const float2* __restrict__ roots, int t) {
    constexpr int NB = P::N / R;
    constexpr int ITEMS = 2 * NB;
    constexpr bool BIG_ODD = (R % 2 == 1 && R > 5);
    constexpr int NS = BIG_ODD ? P::T / ITEMS : 1;   // threads sharing one butterfly
    if constexpr (NS >= 2) {
        // Fewer butterflies than threads: NS threads share each one.  All of
        // them fold the inputs (a_j, b_j); thread s of the group forms the
        // output pairs q = s+1, s+1+NS, ... and thread 0 also the DC term.
        // Every lane takes part, padding lanes too: this stage only reads
        // and writes shared memory.
        constexpr int H = (R - 1) / 2;
        if (t >= NS * ITEMS) return;
        const int f = t % ITEMS, s = t / ITEMS;
        const int i = f >> 1, c = f & 1;
        const int k = i % p;
        const int ob = (i - k) * R + k;
        float2 a[H], b[H];
        const float2 x0 = src[padi(2 * i + c)];
        float2 y0 = x0;
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            float2 u = src[padi(2 * (i + j * NB) + c)];
            float2 w = src[padi(2 * (i + (R - j) * NB) + c)];
            if (p > 1) {
                u = twmul<SIGN>(u, tw[k * (R - 1) + j - 1]);
                w = twmul<SIGN>(w, tw[k * (R - 1) + R - j - 1]);
            }
            a[j - 1] = u + w;
            b[j - 1] = u - w;
            y0 = y0 + a[j - 1];
        }
        if (s == 0) dst[padi(2 * ob + c)] = y0;
        // output pairs with compile-time q: the roots are immediates
        odd_pairs_for<SIGN, R, NS, 0>(s, a, b, x0, dst, ob, p, c);
        (void)roots;
        return;
    }
    if (P::TA != P::T && t >= P::TA) return;   // padding lanes own no element
#pragma unroll
    for (int b = 0; b < (ITEMS + P::TA - 1) / P::TA; ++b) {
        const int f = t + P::TA * b;
        if (ITEMS % P::TA != 0 && f >= ITEMS) break;
        const int i = f >> 1, c = f & 1;
        const int k = i % p;
        const int ob = (i - k) * R + k;
        if constexpr (R % 2 == 1 && R > 5) {
            // large odd radix: fold to a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}
            // and store each output pair as soon as it is formed, so only
            // R - 1 complex values stay live (bfly_odd keeps 3R)
            constexpr int H = (R - 1) / 2;
            float2 a[H], b[H];
            const float2 x0 = src[padi(2 * i + c)];
            float2 y0 = x0;
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                float2 u = src[padi(2 * (i + j * NB) + c)];
                float2 w = src[padi(2 * (i + (R - j) * NB) + c)];
                if (p > 1) {
                    u = twmul<SIGN>(u, tw[k * (R - 1) + j - 1]);
                    w = twmul<SIGN>(w, tw[k * (R - 1) + R - j - 1]);
                }
                a[j - 1] = u + w;
                b[j - 1] = u - w;
                y0 = y0 + a[j - 1];
            }
            dst[padi(2 * ob + c)] = y0;
#pragma unroll
            for (int q = 1; q <= H; ++q) {
                float2 re = x0, im = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 1; j <= H; ++j) {
                    const float2 w = roots[(j * q) % R];
                    re.x += a[j - 1].x * w.x; re.y += a[j - 1].y * w.x;
                    im.x += b[j - 1].x * w.y; im.y += b[j - 1].y * w.y;
                }
                const float2 si = mul_si<SIGN>(im);
                dst[padi(2 * (ob + q * p) + c)] = re + si;
                dst[padi(2 * (ob + (R - q) * p) + c)] = re - si;
            }
        } else {
            float2 v[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                float2 x = src[padi(2 * (i + j * NB) + c)];
                if (j > 0 && p > 1) x = twmul<SIGN>(x, tw[k * (R - 1) + j - 1]);
                v[j] = x;
            }
            bfly<SIGN, R>(v, roots);
#pragma unroll
            for (int j = 0; j < R; ++j) dst[padi(2 * (ob + j * p) + c)] = v[j];
        }
    }
}

// A stage whose inputs are the thread's registers (w[b + j*E/R]); writes its
// outputs to smem (exchange) or, when p*R == N, back into w in place.
template <class P, int SIGN, int R, int p>
__device__ __forceinline__ void stage_reg(float2* w, float2* __restrict__ dst, const float2* __restrict__ tw,
                                          const float2* __restrict__ roots, int t) {
    constexpr int BR = P::E / R;   // butterflies per thread
    constexpr bool LAST = (p * R == P::N);
    if (P::TA != P::T && t >= P::TA) return;
#pragma unroll
    for (int b = 0; b < BR; ++b) {
        const int f = t + P::TA * b;
        const int i = f >> 1, c = f & 1;
        const int k = LAST ? i : (i % p);
        float2 v[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            float2 x = w[b + j * BR];
            if (j > 0 && p > 1) x = twmul<SIGN>(x, tw[k * (R - 1) + j - 1]);
            v[j] = x;
        }
        bfly<SIGN, R>(v, roots);
        if constexpr (LAST) {
#pragma unroll
            for (int j = 0; j < R; ++j) w[b + j * BR] = v[j];
        } else {
            const int ob = (i - k) * R + k;
#pragma unroll
            for (int j = 0; j < R; ++j) dst[padi(2 * (ob + j * p) + c)] = v[j];
        }
    }
}

// Last stage reading smem, writing the thread's registers (p*R == N).
template <class P, int SIGN, int R, int p>
__device__ __forceinline__ void stage_to_reg(const float2* __restrict__ src, float2* w, const float2* __restrict__ tw,
                                             const float2* __restrict__ roots, int t) {
    static_assert(p * R == P::N, "stage_to_reg is the last stage");
    constexpr int NB = P::N / R;
    constexpr int BR = P::E / R;
    if (P::TA != P::T && t >= P::TA) return;
#pragma unroll
    for (int b = 0; b < BR; ++b) {
        const int f = t + P::TA * b;
        const int i = f >> 1, c = f & 1;
        float2 v[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            float2 x = src[padi(2 * (i + j * NB) + c)];
            if (j > 0) x = twmul<SIGN>(x, tw[i * (R - 1) + j - 1]);
            v[j] = x;
        }
        bfly<SIGN, R>(v, roots);
#pragma unroll
        for (int j = 0; j < R; ++j) w[b + j * BR] = v[j];
    }
}

template <class P>
__device__ __forceinline__ void group_sync() {
    if constexpr (P::T == 32) __syncwarp();
    else __syncthreads();
}

// Forward transform: registers (state layout) -> registers (mid layout of
// the last radix).  Stages 0..S-2 go through smem buffers A/B.
template <class P, int s>
__device__ __forceinline__ void fwd_rest(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                         int t) {
    if constexpr (s < P::S) {
        constexpr int R = P::R[s];
        constexpr int p = P::prod(s);
        constexpr int off = Tw<P>::fwd(s);
        float2* src = (s % 2 == 1) ? A : B;
        float2* dst = (s % 2 == 1) ? B : A;
        if constexpr (s == P::S - 1) {
            stage_to_reg<P, -1, R, p>(src, w, tw + off, roots, t);
        } else {
            stage_smem<P, -1, R, p>(src, dst, tw + off, roots, t);
            group_sync<P>();
            fwd_rest<P, s + 1>(w, A, B, tw, roots, t);
        }
    }
}

template <class P>
__device__ __forceinline__ void forward(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                        int t) {
    constexpr int R0 = P::R[0];
    if constexpr (P::S == 1) {
        stage_reg<P, -1, R0, 1>(w, nullptr, tw, roots, t);
    } else {
        stage_reg<P, -1, R0, 1>(w, A, tw, roots, t);   // outputs to A
        group_sync<P>();
        fwd_rest<P, 1>(w, A, B, tw, roots, t);
    }
}

// Inverse transform: registers (mid layout of R[S-1]) -> registers (state).
template <class P, int s>
__device__ __forceinline__ void inv_rest(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                         int t) {
    if constexpr (s < P::S) {
        constexpr int R = P::R[P::S - 1 - s];
        constexpr int p = P::rprod(s);
        constexpr int off = Tw<P>::inv(s);
        float2* src = (s % 2 == 1) ? A : B;
        float2* dst = (s % 2 == 1) ? B : A;
        if constexpr (s == P::S - 1) {
            stage_to_reg<P, +1, R, p>(src, w, tw + off, roots, t);
        } else {
            stage_smem<P, +1, R, p>(src, dst, tw + off, roots, t);
            group_sync<P>();
            inv_rest<P, s + 1>(w, A, B, tw, roots, t);
        }
    }
}

template <class P>
__device__ __forceinline__ void inverse(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                        int t) {
    constexpr int R0 = P::R[P::S - 1];
    if constexpr (P::S == 1) {
        stage_reg<P, +1, R0, 1>(w, nullptr, tw + Tw<P>::inv(0), roots, t);
    } else {
        stage_reg<P, +1, R0, 1>(w, A, tw + Tw<P>::inv(0), roots, t);
        group_sync<P>();
        inv_rest<P, 1>(w, A, B, tw, roots, t);
    }
}

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

__device__ __forceinline__ float2 shrink_c(float2 c, float lam) {
    const float m = sqrtf(c.x * c.x + c.y * c.y);   // wavelet.rs:90 |z|
    if (m <= lam) return make_float2(0.f, 0.f);
    return c * ((m - lam) / m);
}

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
    __syncthreads();
    const int nrp = a.ny / 2;
    const bool live = t < TA;
    const float alpha = mode ? __ldg(a.alpha + it) : 0.f;
    const float lam = a.lambda;
    const bool b0 = (t & 1) != 0, b1 = (t & 2) != 0;
    const long long total = a.nprob * nrp, stride = (long long)gridDim.x * G;
    // pipelined form (a.prefetch bit 1): the next unit's S, Z~, X~ are copied
    // (cp.async) into this thread's own shared-memory slots while the current
    // unit's transforms run
    float2* PF = RT + roots_total + G * 2 * P::SMEM_X + g * 3 * E * T;   // [E][T] S, Z~, X~
    auto issue = [&](long long u) {
        const long long p = u / nrp;
        const int r0 = 2 * (int)(u - p * nrp);
        const uint32_t* cb = a.colbits + ((p + a.mask_offset) % a.mask_mod) * a.col_wstride;
        const long long base = p * a.st_stride + (long long)r0 * N;
        const float2* S = a.S + base;
        const float2* X = a.X + base;
        const float2* Z = a.Z + base;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = t + TA * e;
            const int x = q >> 1;
            const long long off = (long long)(q & 1) * N + x;
            const bool on = live && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u);
            cp_async8(PF + e * T + t, on ? S + off : S, on ? 8u : 0u);
            if (mode) {
                cp_async8(PF + (E + e) * T + t, live ? Z + off : Z, live ? 8u : 0u);
                cp_async8(PF + (2 * E + e) * T + t, live ? X + off : X, live ? 8u : 0u);
            }
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
                const int x = (t + TA * e) >> 1;
                if (live && ((__ldg(cb + (x >> 5)) >> (x & 31)) & 1u)) cm |= 1u << e;
                w[e] = PF[e * T + t];
                zo[e] = mode ? PF[(E + e) * T + t] : make_float2(0.f, 0.f);
                xo[e] = mode ? PF[(2 * E + e) * T + t] : make_float2(0.f, 0.f);
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
using P256 = Plan<256, 32, 16, 16>;
using P320 = Plan<320, 64, 10, 16, 2>;
using P368 = Plan<368, 92, 4, 23, 4>;
using P384 = Plan<384, 64, 12, 8, 4>;
using P192 = Plan<192, 32, 12, 4, 4>;
using P128 = Plan<128, 32, 8, 2, 8>;
using P512 = Plan<512, 64, 16, 2, 16>;
using P640 = Plan<640, 160, 8, 10, 8>;

template <class P>
static cudaError_t plan_tables(const float2** tw, const float2** roots, int* nroots);

// Minimum resident CTAs per SM for the 12-warp occupancy form of the 2-D
// passes (a.occ = 1); the register budget per thread follows from it.
template <class P>
constexpr int occ_blocks() {
    constexpr int threads = P::T * (P::T == 32 ? 4 : 1);
    return (12 * 32 + threads - 1) / threads;
}

template <class P, int MINB>
static cudaError_t launch_2d_k(const Fista2dArgs& a, long long units, cudaStream_t st, int mode, int it, bool row) {
    constexpr int NTW = Tw<P>::total();
    constexpr int G = (P::T == 32) ? 4 : 1;
    const float2 *tw, *rt;
    int nrt;
    cudaError_t e = plan_tables<P>(&tw, &rt, &nrt);
    if (e != cudaSuccess) return e;
    // the pipelined column pass (separable masks) adds each group's prefetch slots
    // and the pipelined row pass its three
    // (left out where they would cost resident CTAs below MINB per SM)
    Fista2dArgs b = a;
    const size_t base_smem = sizeof(float2) * (NTW + nrt + (size_t)G * 2 * P::SMEM_X);
    const size_t pf_smem = sizeof(float2) * (size_t)G * (row ? 3 : 2) * P::E * P::T;
    int pf = row ? ((a.prefetch & 2) ? 1 : 0) : ((a.separable && (a.prefetch & 1)) ? 1 : 0);
    if (pf && MINB > 1 && (base_smem + pf_smem + 1024) * MINB > 220u * 1024u) pf = 0;
    b.prefetch = pf;
    const size_t smem = base_smem + (pf ? pf_smem : 0);
    if (row) e = set_smem_attr(reinterpret_cast<const void*>(k2d_row_reg<P, MINB>), smem);
    else e = set_smem_attr(reinterpret_cast<const void*>(k2d_col_reg<P, MINB>), smem);
    if (e != cudaSuccess) return e;
    long long grid = (units + G - 1) / G;
    // persistent form: every resident CTA slot once, units grid-strided
    // (the kernels accept any grid)
    if (a.persist) {
        static int per_sm[2][2] = {{0, 0}, {0, 0}}, nsm = 0;
        if (!per_sm[row][pf]) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (row) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1][pf], k2d_row_reg<P, MINB>, P::T * G, smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0][pf], k2d_col_reg<P, MINB>, P::T * G, smem);
            if (per_sm[row][pf] < 1) per_sm[row][pf] = 1;
        }
        if (grid > (long long)per_sm[row][pf] * nsm) grid = (long long)per_sm[row][pf] * nsm;
    }
    if (row)
        k2d_row_reg<P, MINB><<<(unsigned)grid, P::T * G, smem, st>>>(b, mode, it, tw, rt, nrt);
    else
        k2d_col_reg<P, MINB><<<(unsigned)grid, P::T * G, smem, st>>>(b, mode, tw, rt, nrt);
    return cudaGetLastError();
}

template <class P>
static cudaError_t launch_2d(const Fista2dArgs& a, long long units, cudaStream_t st, int mode, int it, bool row) {
    if (a.occ) return launch_2d_k<P, occ_blocks<P>()>(a, units, st, mode, it, row);
    return launch_2d_k<P, 1>(a, units, st, mode, it, row);
}

template <class P>
static cudaError_t col2d(const Fista2dArgs& a, RegTables& tabs, int mode, cudaStream_t st) {
    (void)tabs;
    return launch_2d<P>(a, a.nprob * (a.nx / 2), st, mode, 0, false);
}
template <class P>
static cudaError_t row2d(const Fista2dArgs& a, RegTables& tabs, int mode, int it, cudaStream_t st) {
    (void)tabs;
    return launch_2d<P>(a, a.nprob * (a.ny / 2), st, mode, it, true);
}

template <class P>
static void host_tables(float2* tw, int* ntw) {
    const double two_pi = 6.283185307179586476925286766559;
    int o = 0;
    for (int s = 0; s < P::S; ++s) {
        const int R = P::R[s], p = P::prod(s);
        for (int k = 0; k < p; ++k)
            for (int j = 1; j < R; ++j) {
                const double ang = -two_pi * j * k / ((double)p * R);
                tw[o++] = make_float2((float)cos(ang), (float)sin(ang));
            }
    }
    for (int s = 0; s < P::S; ++s) {
        const int R = P::R[P::S - 1 - s], p = P::rprod(s);
        for (int k = 0; k < p; ++k)
            for (int j = 1; j < R; ++j) {
                const double ang = -two_pi * j * k / ((double)p * R);
                tw[o++] = make_float2((float)cos(ang), (float)sin(ang));
            }
    }
    *ntw = o;
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
// E = 8 plans: the SENSE kernel holds five register arrays per element
using S128 = Plan<128, 32, 8, 2, 8>;
using S192 = Plan<192, 48, 8, 3, 8>;
using S256 = Plan<256, 64, 8, 4, 8>;
using S320 = Plan<320, 64, 10, 16, 2>;
using S368 = Plan<368, 92, 4, 23, 4>;
using S384 = Plan<384, 96, 8, 6, 8>;
using S512 = Plan<512, 128, 8, 8, 8>;

// Twiddle / root tables of plan P on the current device, built on first use
// and kept for the life of the process (a few KB per plan and device).
template <class P>
static cudaError_t plan_tables(const float2** tw, const float2** roots, int* nroots) {
    static float2* d_tab[64] = {};
    static int d_nrt[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!d_tab[dev]) {
        static float2 h[4096 + 64];
        int ntw = 0;
        host_tables<P>(h, &ntw);
        int nrt = 1;
        h[ntw] = make_float2(1.f, 0.f);
        for (int s = 0; s < P::S; ++s)
            if (P::R[s] % 2 == 1 && P::R[s] > 5) {   // generic odd radix: (cos, sin)(2 pi m / R)
                nrt = P::R[s];
                for (int m = 0; m < nrt; ++m) {
                    const double ang = 6.283185307179586476925286766559 * m / nrt;
                    h[ntw + m] = make_float2((float)cos(ang), (float)sin(ang));
                }
            }
        float2* d = nullptr;
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * (ntw + nrt));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h, sizeof(float2) * (ntw + nrt), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        d_tab[dev] = d;
        d_nrt[dev] = nrt;
    }
    *tw = d_tab[dev];
    *roots = d_tab[dev] + Tw<P>::total();
    *nroots = d_nrt[dev];
    return cudaSuccess;
}

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

int fista_col_reg_variants(int ny) { return (ny == 192 || ny == 256 || ny == 384 || ny == 512) ? 2 : 1; }

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
