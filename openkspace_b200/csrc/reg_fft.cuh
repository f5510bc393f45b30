// Register-resident Stockham FFT building blocks shared by the sm_100a
// kernels that keep a column pair or row pair of one problem in registers
// (k_fista_reg.cu: FISTA engines; k_xform_reg.cu: standalone transforms).
//
// A plan Plan<N, TA, R0, R1, ...> runs a length-N transform of two
// interleaved lines (element q = 2 * index + line) on TA active threads;
// thread t holds elements q = t + TA * e, e < E = 2N / TA, in natural
// order both before and after forward<P> / inverse<P>.  Intermediate
// stages exchange through two shared-memory buffers per thread group.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "fft_dev.cuh"
#include "kernels.h"

// Bounds-checked build (-DOKS_BOUNDS_CHECK, libokscuda_bounds.so): every
// exchange-buffer and staging-buffer index is range-checked before use; an
// index out of range sets a bit of a device error word (one per translation
// unit, read through okscuda_debug_bounds) and the access is skipped.  No
// assert and no trap: the kernel runs on and returns.  In the normal build
// OKS_IN is the constant true and the checks compile away.
#ifdef OKS_BOUNDS_CHECK
namespace oks {
static __device__ unsigned int g_bounds_word;
__device__ __forceinline__ bool bounds_ok(long long i, long long n, unsigned code) {
    if (i >= 0 && i < n) return true;
    atomicOr(&g_bounds_word, code);
    return false;
}
// Host side: this translation unit's word, read (and cleared) by
// okscuda_debug_bounds through a registry defined in api.cu.
void bounds_register(unsigned (*reader)(int clear));
namespace {
unsigned bounds_read_tu(int clear) {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_bounds_word, sizeof v) != cudaSuccess) return 0x80000000u;
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_bounds_word, &z, sizeof z);
    }
    return v;
}
struct BoundsRegistrar {
    BoundsRegistrar() { bounds_register(&bounds_read_tu); }
};
static BoundsRegistrar g_bounds_registrar;
}  // namespace
}  // namespace oks
#define OKS_IN(i, n, code) ::oks::bounds_ok((long long)(i), (long long)(n), (code))
#else
#define OKS_IN(i, n, code) true
#endif
// Error-word bits of the bounds-checked build.
#define OKS_B_XCHG 1u      // exchange buffer (logical index outside [0, 2N))
#define OKS_B_STAGE 2u     // staging / prefetch buffer
#define OKS_B_TILE 4u      // column tile (lanes form)

namespace oks {
namespace reg {


// Exchange-buffer index: an XOR swizzle inside each aligned block of 16
// float2 (one 128-byte row of banks).  The Stockham writes stride by 2R
// elements across lanes; folding bits 3.. and 6.. of the index into the low
// four bits spreads those strides over all 16 8-byte bank slots.  A bank model
// of every stage of every plan gives 1.00-1.31x the conflict-free wavefront
// count (the former "+1 float2 per 32" padding: 1.25-1.75x).
__device__ __forceinline__ int padi(int i) { return i ^ (((i >> 3) ^ (i >> 6)) & 15); }

// Second exchange layout, one pad per 16 entries: lin16(v) = v + v / 16.  It
// is linear in steps of 16, so a stage reading x[i + j N/R] with 2 N/R a
// multiple of 16 addresses every j as one base plus a compile-time offset
// (padi costs about five integer operations per access).  Stores of a first
// stage of radix 4, 8 or 16 (lanes 2R apart) fall on distinct bank pairs in
// it, so the buffer between the first and the second stage uses it.
__device__ __forceinline__ int lin16(int v) { return v + (v >> 4); }

// Source index of element (i + j NB, c) in the padi or the lin16 layout.
template <bool LIN, int NB>
struct SrcIdx {
    int base;
    __device__ __forceinline__ SrcIdx(int i, int c) : base(LIN ? lin16(2 * i + c) : 2 * i + c) {}
    __device__ __forceinline__ int operator()(int j) const {
        if constexpr (LIN) return base + j * (2 * NB + (2 * NB) / 16);
        else return padi(base + 2 * j * NB);
    }
};

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
    // exchange buffer (float2): padi keeps every index below 2N rounded up
    // to 16, lin16 below 2N + 2N/16
    static constexpr int SMEM_X = 2 * N_ + (2 * N_) / 16 + 1;
    // largest index each layout writes: padi stays inside the aligned block
    // of 16 of its argument (< 2N rounded up to 16), lin16 reaches lin16(2N - 1)
    static constexpr int PADI_END = (2 * N_ + 15) / 16 * 16;
    static constexpr int LIN16_END = (2 * N_ - 1) + (2 * N_ - 1) / 16 + 1;
    static_assert(PADI_END <= SMEM_X, "padi exchange indices overrun the buffer");
    static_assert(LIN16_END <= SMEM_X, "lin16 exchange indices overrun the buffer");
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
// PRE: the inputs already carry this stage's twiddles (the previous stage
// applied them as it stored, once per element; only for the split form).
// LIN: src is in the lin16 layout (written by a first stage with LINW).
template <class P, int SIGN, int R, int p, bool PRE = false, bool LIN = false>
__device__ __forceinline__ void stage_smem(const float2* __restrict__ src, float2* __restrict__ dst,
                                           const float2* __restrict__ tw, const float2* __restrict__ roots, int t) {
    constexpr int NB = P::N / R;
    static_assert(!LIN || (2 * NB) % 16 == 0, "lin16 reads need 2 N/R to be a multiple of 16");
    constexpr int ITEMS = 2 * NB;
    constexpr bool BIG_ODD = (R % 2 == 1 && R > 5);
    constexpr int NS = BIG_ODD ? P::T / ITEMS : 1;   // threads sharing one butterfly
    static_assert(!PRE || NS >= 2, "pre-twiddled inputs are for the split odd-radix form");
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
        const SrcIdx<LIN, NB> ix(i, c);
        if (!OKS_IN(2 * (i + (R - 1) * NB) + c, 2 * P::N, OKS_B_XCHG)) return;
        const float2 x0 = src[ix(0)];
        float2 y0 = x0;
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            float2 u = src[ix(j)];
            float2 w = src[ix(R - j)];
            if (p > 1 && !PRE) {
                u = twmul<SIGN>(u, tw[k * (R - 1) + j - 1]);
                w = twmul<SIGN>(w, tw[k * (R - 1) + R - j - 1]);
            }
            a[j - 1] = u + w;
            b[j - 1] = u - w;
            y0 = y0 + a[j - 1];
        }
        if (!OKS_IN(2 * (ob + (R - 1) * p) + c, 2 * P::N, OKS_B_XCHG)) return;
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
            const SrcIdx<LIN, NB> ix(i, c);
            if (!OKS_IN(2 * (i + (R - 1) * NB) + c, 2 * P::N, OKS_B_XCHG) ||
                !OKS_IN(2 * (ob + (R - 1) * p) + c, 2 * P::N, OKS_B_XCHG))
                continue;
            const float2 x0 = src[ix(0)];
            float2 y0 = x0;
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                float2 u = src[ix(j)];
                float2 w = src[ix(R - j)];
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
            const SrcIdx<LIN, NB> ix(i, c);
            if (!OKS_IN(2 * (i + (R - 1) * NB) + c, 2 * P::N, OKS_B_XCHG) ||
                !OKS_IN(2 * (ob + (R - 1) * p) + c, 2 * P::N, OKS_B_XCHG))
                continue;
#pragma unroll
            for (int j = 0; j < R; ++j) {
                float2 x = src[ix(j)];
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
// R2 > 0: the next stage (radix R2, P2 = p R) is the split odd-radix form;
// each output o = i2 + j2 N/R2 is stored already multiplied by that stage's
// twiddle w^(j2 k2), k2 = i2 mod P2 (tw2: its table), so the NS threads
// sharing a butterfly there do not each repeat the 2 (R2 - 1) products.  The
// products are the same, so the results are bit-identical.
// LINW: store in the lin16 layout (the next stage reads with LIN).
template <class P, int SIGN, int R, int p, int R2 = 0, int P2 = 0, bool LINW = false>
__device__ __forceinline__ void stage_reg(float2* w, float2* __restrict__ dst, const float2* __restrict__ tw,
                                          const float2* __restrict__ roots, int t,
                                          const float2* __restrict__ tw2 = nullptr) {
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
            for (int j = 0; j < R; ++j) {
                float2 y = v[j];
                if constexpr (R2 > 0) {
                    constexpr int NB2 = P::N / R2;
                    const int o = ob + j * p;
                    const int j2 = o / NB2, k2 = (o - j2 * NB2) % P2;
                    if (j2 > 0 && k2 > 0) y = twmul<SIGN>(y, tw2[k2 * (R2 - 1) + j2 - 1]);
                }
                const int v = 2 * (ob + j * p) + c;
                if (OKS_IN(v, 2 * P::N, OKS_B_XCHG)) dst[LINW ? lin16(v) : padi(v)] = y;
            }
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
            float2 x = OKS_IN(2 * (i + j * NB) + c, 2 * P::N, OKS_B_XCHG) ? src[padi(2 * (i + j * NB) + c)]
                                                                           : make_float2(0.f, 0.f);
            if (j > 0) x = twmul<SIGN>(x, tw[i * (R - 1) + j - 1]);
            v[j] = x;
        }
        bfly<SIGN, R>(v, roots);
#pragma unroll
        for (int j = 0; j < R; ++j) w[b + j * BR] = v[j];
    }
}

// True when the buffer between the first and the second stage of a direction
// (first radix R0, second R1) takes the lin16 layout: a plan of 3 or more
// stages, R0 in {4, 8, 16}, 2 N/R1 a multiple of 16.  The drivers' L = false
// keeps padi throughout (the tiled column transform ran 5-7 % slower at 384
// and 640 with lin16, while the row transforms ran 8-16 % faster).
template <class P, int R0, int R1>
constexpr bool lin_first() {
    return P::S >= 3 && (R0 == 4 || R0 == 8 || R0 == 16) && R1 > 0 && (2 * (P::N / R1)) % 16 == 0;
}
template <class P>
constexpr bool lin_fwd() { return lin_first<P, P::R[0], (P::S >= 2 ? P::R[P::S >= 2 ? 1 : 0] : 0)>(); }
template <class P>
constexpr bool lin_inv() { return lin_first<P, P::R[P::S - 1], (P::S >= 2 ? P::R[P::S >= 2 ? P::S - 2 : 0] : 0)>(); }

// True when a middle stage of radix R runs in the split odd-radix form (the
// plan has fewer of its butterflies than threads).
template <class P, int R>
constexpr bool split_odd_stage() {
    return R % 2 == 1 && R > 5 && P::T / (2 * (P::N / R)) >= 2;
}

// Barrier of one thread group.  NB (named barriers): groups of T >= 64
// threads that share a CTA wait on barrier 1 + group index only, so the
// groups do not hold each other up stage by stage.
template <class P, bool NB = false>
__device__ __forceinline__ void group_sync() {
    if constexpr (P::T == 32) {
        __syncwarp();
    } else if constexpr (NB) {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / P::T)), "n"(P::T) : "memory");
    } else {
        __syncthreads();
    }
}

// Forward transform: registers (state layout) -> registers (mid layout of
// the last radix).  Stages 0..S-2 go through smem buffers A/B.
template <class P, int s, bool NB = false, bool L = true>
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
            constexpr bool PRE = s == 1 && split_odd_stage<P, R>();   // twiddled by stage 0's stores
            stage_smem<P, -1, R, p, PRE, L && s == 1 && lin_fwd<P>()>(src, dst, tw + off, roots, t);
            group_sync<P, NB>();
            fwd_rest<P, s + 1, NB, L>(w, A, B, tw, roots, t);
        }
    }
}

template <class P, bool NB = false, bool L = true>
__device__ __forceinline__ void forward(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                        int t) {
    constexpr int R0 = P::R[0];
    if constexpr (P::S == 1) {
        stage_reg<P, -1, R0, 1>(w, nullptr, tw, roots, t);
    } else {
        if constexpr (P::S >= 3 && split_odd_stage<P, P::R[1]>())
            stage_reg<P, -1, R0, 1, P::R[1], R0, L && lin_fwd<P>()>(w, A, tw, roots, t, tw + Tw<P>::fwd(1));
        else
            stage_reg<P, -1, R0, 1, 0, 0, L && lin_fwd<P>()>(w, A, tw, roots, t);   // outputs to A
        group_sync<P, NB>();
        fwd_rest<P, 1, NB, L>(w, A, B, tw, roots, t);
    }
}

// Inverse transform: registers (mid layout of R[S-1]) -> registers (state).
template <class P, int s, bool NB = false, bool L = true>
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
            constexpr bool PRE = s == 1 && split_odd_stage<P, R>();   // twiddled by stage 0's stores
            stage_smem<P, +1, R, p, PRE, L && s == 1 && lin_inv<P>()>(src, dst, tw + off, roots, t);
            group_sync<P, NB>();
            inv_rest<P, s + 1, NB, L>(w, A, B, tw, roots, t);
        }
    }
}

template <class P, bool NB = false, bool L = true>
__device__ __forceinline__ void inverse(float2* w, float2* A, float2* B, const float2* tw, const float2* roots,
                                        int t) {
    constexpr int R0 = P::R[P::S - 1];
    if constexpr (P::S == 1) {
        stage_reg<P, +1, R0, 1>(w, nullptr, tw + Tw<P>::inv(0), roots, t);
    } else {
        if constexpr (P::S >= 3 && split_odd_stage<P, P::R[P::S - 2]>())
            stage_reg<P, +1, R0, 1, P::R[P::S - 2], R0, L && lin_inv<P>()>(w, A, tw + Tw<P>::inv(0), roots, t,
                                                                  tw + Tw<P>::inv(1));
        else
            stage_reg<P, +1, R0, 1, 0, 0, L && lin_inv<P>()>(w, A, tw + Tw<P>::inv(0), roots, t);
        group_sync<P, NB>();
        inv_rest<P, 1, NB, L>(w, A, B, tw, roots, t);
    }
}

// Programmatic dependent launch: pdl_wait() returns once the grid this one
// depends on in its stream has completed and its writes are visible (at once
// for a grid launched without the attribute); pdl_trigger() lets the next
// grid of the stream be scheduled (its CTAs take SM slots as this grid's CTAs
// leave, and run their prologue up to their own pdl_wait).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}


// Register plans: N, active threads, radices.
using P256 = Plan<256, 32, 16, 16>;
using P320 = Plan<320, 64, 10, 16, 2>;
using P368 = Plan<368, 92, 4, 23, 4>;
using P384 = Plan<384, 64, 12, 8, 4>;
using P192 = Plan<192, 32, 12, 4, 4>;
using P128 = Plan<128, 32, 8, 2, 8>;
using P512 = Plan<512, 64, 16, 2, 16>;
using P640 = Plan<640, 160, 8, 10, 8>;

// E = 8 plans: the SENSE kernel holds five register arrays per element
using S128 = Plan<128, 32, 8, 2, 8>;
using S192 = Plan<192, 48, 8, 3, 8>;
using S256 = Plan<256, 64, 8, 4, 8>;
using S320 = Plan<320, 64, 10, 16, 2>;
using S368 = Plan<368, 92, 4, 23, 4>;
using S384 = Plan<384, 96, 8, 6, 8>;
using S512 = Plan<512, 128, 8, 8, 8>;
// E = 8 alternative for 320 (80 active threads of 96)
using V320 = Plan<320, 80, 8, 5, 8>;

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

// Host image of plan P's device tables: the twiddles (host_tables order)
// followed by the roots of its generic odd radix (or one unit root).  Writes
// Tw<P>::total() + *nroots entries to h (at most 4096 + 64).
template <class P>
static int host_plan_tables(float2* h, int* nroots) {
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
    *nroots = nrt;
    return ntw + nrt;
}

// Twiddle / root tables of plan P on the current device, built on first use
// and kept for the life of the process (a few KB per plan and device).
template <class P>
static cudaError_t plan_tables(const float2** tw, const float2** roots, int* nroots) {
    static float2* d_tab[64] = {};
    static int d_nrt[64] = {};
    static std::mutex mu;   // contexts on different host threads may build a plan's tables at once
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!d_tab[dev]) {
        static float2 h[4096 + 64];
        int nrt = 1;
        const int total = host_plan_tables<P>(h, &nrt);
        float2* d = nullptr;
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * total);
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h, sizeof(float2) * total, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        d_tab[dev] = d;
        d_nrt[dev] = nrt;
    }
    *tw = d_tab[dev];
    *roots = d_tab[dev] + Tw<P>::total();
    *nroots = d_nrt[dev];
    return cudaSuccess;
}


}  // namespace reg
}  // namespace oks
