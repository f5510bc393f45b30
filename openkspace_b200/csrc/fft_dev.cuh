// Device-side FFT building blocks for sm_100a: complex helpers, radix-R
// butterflies and a Stockham autosort stage over shared memory.
//
// Conventions.  SIGN = -1 is the forward DFT (e^{-2 pi i jk/n}), SIGN = +1
// the unnormalised inverse.  A Stockham stage of radix R with p = product of
// the earlier radices takes butterfly i in [0, n/R), k = i mod p, inputs
// x[i + j n/R] * w_{pR}^{jk}, an R-point DFT, and writes y[(i-k)R + k + jp].
// After all stages the output is in natural order.  Twiddle tables are built
// on the host in double precision for the forward sign; the inverse uses
// their conjugates.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace oks {

__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// wavelet.rs:90-96 soft threshold: |z| <= lambda -> 0, else z (|z| - lambda) / |z|.
// shrink_c writes it as z (1 - lambda / |z|) with the reciprocal square root
// of |z|^2 (one multi-function-unit op and two FMAs in place of a square root
// and a division; |z| <= lambda is |z|^2 <= lambda^2 for lambda >= 0).  The
// register FISTA engines use it: 16-21 % more slices/s on B200.
// shrink_exact keeps the reference's square root and division.  It is used in
// the separate prox kernel of the tensor-core row engine, which ran 25 % fewer
// slices/s with shrink_c on B200, and in the shared-memory fallbacks and the
// soft-threshold primitive.
__device__ __forceinline__ float2 shrink_c(float2 c, float lam) {
    const float m2 = c.x * c.x + c.y * c.y;
    if (lam >= 0.f && m2 <= lam * lam) return make_float2(0.f, 0.f);
    return c * (1.f - lam * rsqrtf(m2));
}
__device__ __forceinline__ float2 shrink_exact(float2 c, float lam) {
    const float m = sqrtf(c.x * c.x + c.y * c.y);
    if (m <= lam) return make_float2(0.f, 0.f);
    return c * ((m - lam) / m);
}

template <int SIGN>
__device__ __forceinline__ float2 twmul(float2 a, float2 w) {
    return SIGN < 0 ? cmul(a, w) : cmulc(a, w);
}
// SIGN * i * a
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 a) {
    return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// ---------------------------------------------------------------- butterflies
template <int SIGN>
__device__ __forceinline__ void bfly2(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}

template <int SIGN>
__device__ __forceinline__ void bfly3(float2* v) {
    const float s3 = 0.86602540378443864676f;
    float2 t1 = v[1] + v[2];
    float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 t3 = mul_si<SIGN>(v[1] - v[2]) * s3;
    v[0] = v[0] + t1;
    v[1] = t2 + t3;
    v[2] = t2 - t3;
}

template <int SIGN>
__device__ __forceinline__ void bfly4(float2* v) {
    float2 a = v[0] + v[2], b = v[0] - v[2];
    float2 c = v[1] + v[3], d = mul_si<SIGN>(v[1] - v[3]);
    v[0] = a + c;
    v[1] = b + d;
    v[2] = a - c;
    v[3] = b - d;
}

template <int SIGN>
__device__ __forceinline__ void bfly5(float2* v) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 a1 = v[1] + v[4], b1 = v[1] - v[4];
    float2 a2 = v[2] + v[3], b2 = v[2] - v[3];
    float2 x0 = v[0];
    float2 t1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    float2 t2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    float2 u1 = mul_si<SIGN>(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    float2 u2 = mul_si<SIGN>(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = x0 + a1 + a2;
    v[1] = t1 + u1;
    v[4] = t1 - u1;
    v[2] = t2 + u2;
    v[3] = t2 - u2;
}

template <int SIGN>
__device__ __forceinline__ void bfly8(float2* v) {
    const float h = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    bfly4<SIGN>(e);
    bfly4<SIGN>(o);
    // w8^1 = h (1 + SIGN i), w8^2 = SIGN i, w8^3 = h (-1 + SIGN i)
    float2 o1 = (o[1] + mul_si<SIGN>(o[1])) * h;
    float2 o2 = mul_si<SIGN>(o[2]);
    float2 o3 = (mul_si<SIGN>(o[3]) - o[3]) * h;
    v[0] = e[0] + o[0]; v[4] = e[0] - o[0];
    v[1] = e[1] + o1;   v[5] = e[1] - o1;
    v[2] = e[2] + o2;   v[6] = e[2] - o2;
    v[3] = e[3] + o3;   v[7] = e[3] - o3;
}

template <int SIGN>
__device__ __forceinline__ void bfly16(float2* v) {
    float2 e[8], o[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { e[q] = v[2 * q]; o[q] = v[2 * q + 1]; }
    bfly8<SIGN>(e);
    bfly8<SIGN>(o);
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    // w16^k = cos(2 pi k/16) + SIGN i sin(2 pi k/16)
    const float cs[8] = {1.f, c1, h, s1, 0.f, -s1, -h, -c1};
    const float sn[8] = {0.f, s1, h, c1, 1.f, c1, h, s1};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float2 w = make_float2(cs[k], SIGN * sn[k]);
        float2 t = cmul(o[k], w);
        v[k] = e[k] + t;
        v[k + 8] = e[k] - t;
    }
}

// Odd radix R (any), symmetric form: for q in 1..(R-1)/2
//   y_q     = x0 + sum_j a_j cos(2 pi jq/R) + SIGN i sum_j b_j sin(2 pi jq/R)
//   y_{R-q} = x0 + sum_j a_j cos(...)       - SIGN i sum_j b_j sin(...)
// with a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}.  `cs` holds cos/sin of
// 2 pi m / R for m in [0, R) as float2(cos, sin).
template <int SIGN, int R>
__device__ __forceinline__ void bfly_odd(float2* v, const float2* __restrict__ cs) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
    float2 y0 = v[0];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
        a[j - 1] = v[j] + v[R - j];
        b[j - 1] = v[j] - v[R - j];
        y0 = y0 + a[j - 1];
    }
    float2 out[R];
    out[0] = y0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
        float2 re = v[0], im = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            float2 w = cs[(j * q) % R];
            re.x += a[j - 1].x * w.x; re.y += a[j - 1].y * w.x;
            im.x += b[j - 1].x * w.y; im.y += b[j - 1].y * w.y;
        }
        float2 si = mul_si<SIGN>(im);
        out[q] = re + si;
        out[R - q] = re - si;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

// ------------------------------------------------------------ stage plans
constexpr int kMaxStages = 24;

// One FFT length: forward stages with radices rad[0..nst), their p and twiddle
// offsets; the matching inverse plan uses the reversed radix order (so that
// its first stage reads exactly the outputs of the forward plan's last
// butterflies).  Twiddle tables (float2, forward sign) live in global memory:
//   tw[off + k*(R-1) + j-1] = w_{pR}^{jk};   roots[roff + m] = (cos, sin)(2 pi m/R)
struct FftPlan {
    int n;
    int nst;
    int rad[kMaxStages];
    int p_f[kMaxStages], tw_f[kMaxStages];   // forward order
    int p_i[kMaxStages], tw_i[kMaxStages];   // reversed order (stage s uses rad[nst-1-s])
    int root_off[kMaxStages];                // per forward stage index (same radix either way)
    int tw_total;                            // float2 entries in the table
};

// Generic smem stage: `nl` independent lanes of length n; element (lane, idx)
// at lane * ls + idx * es.  Work items are (lane, butterfly) pairs; with
// LANE_FAST the lane index varies fastest across threads.
template <int SIGN, bool LANE_FAST>
__device__ void stage_smem(const float2* __restrict__ src, float2* __restrict__ dst,
                           int n, int R, int p, const float2* __restrict__ tw,
                           const float2* __restrict__ roots, int nl, int ls, int es,
                           int tid, int nthr) {
    const int nb = n / R;
    const int total = nb * nl;
    for (int f = tid; f < total; f += nthr) {
        int lane, i;
        if (LANE_FAST) { lane = f % nl; i = f / nl; }
        else           { i = f % nb; lane = f / nb; }
        const int k = i % p;
        const int ob = (i - k) * R + k;
        const float2* s = src + lane * ls;
        float2* d = dst + lane * ls;
        const float2* t = tw + k * (R - 1);
#define OKS_LOAD(RR)                                                   \
    float2 v[RR];                                                      \
    v[0] = s[i * es];                                                  \
    _Pragma("unroll") for (int j = 1; j < RR; ++j)                     \
        v[j] = twmul<SIGN>(s[(i + j * nb) * es], t[j - 1]);
#define OKS_STORE(RR)                                                  \
    _Pragma("unroll") for (int j = 0; j < RR; ++j) d[(ob + j * p) * es] = v[j];
        switch (R) {
            case 2: { OKS_LOAD(2) bfly2<SIGN>(v); OKS_STORE(2) } break;
            case 3: { OKS_LOAD(3) bfly3<SIGN>(v); OKS_STORE(3) } break;
            case 4: { OKS_LOAD(4) bfly4<SIGN>(v); OKS_STORE(4) } break;
            case 5: { OKS_LOAD(5) bfly5<SIGN>(v); OKS_STORE(5) } break;
            case 8: { OKS_LOAD(8) bfly8<SIGN>(v); OKS_STORE(8) } break;
            case 16: { OKS_LOAD(16) bfly16<SIGN>(v); OKS_STORE(16) } break;
            case 7: { OKS_LOAD(7) bfly_odd<SIGN, 7>(v, roots); OKS_STORE(7) } break;
            case 11: { OKS_LOAD(11) bfly_odd<SIGN, 11>(v, roots); OKS_STORE(11) } break;
            case 13: { OKS_LOAD(13) bfly_odd<SIGN, 13>(v, roots); OKS_STORE(13) } break;
            case 17: { OKS_LOAD(17) bfly_odd<SIGN, 17>(v, roots); OKS_STORE(17) } break;
            case 19: { OKS_LOAD(19) bfly_odd<SIGN, 19>(v, roots); OKS_STORE(19) } break;
            case 23: { OKS_LOAD(23) bfly_odd<SIGN, 23>(v, roots); OKS_STORE(23) } break;
            default: {
                // any other radix: direct DFT, inputs re-read from smem
                for (int q = 0; q < R; ++q) {
                    float2 acc = s[i * es];
                    for (int j = 1; j < R; ++j) {
                        float2 x = twmul<SIGN>(s[(i + j * nb) * es], t[j - 1]);
                        // roots hold (cos, sin)(2 pi m/R); forward uses e^{-i theta}
                        float2 w = roots[(int)(((long long)j * q) % R)];
                        float2 e = SIGN < 0 ? make_float2(w.x, -w.y) : w;
                        acc = acc + cmul(x, e);
                    }
                    d[(ob + q * p) * es] = acc;
                }
            } break;
        }
#undef OKS_LOAD
#undef OKS_STORE
    }
}

// Run every stage of a plan over smem.  Reads `src` (left untouched unless
// it is one of the two work buffers), ping-pongs between bufA and bufB, and
// returns the buffer holding the natural-order result.  Ends with a barrier.
template <int SIGN, bool LANE_FAST>
__device__ float2* fft_smem(const float2* src, float2* bufA, float2* bufB, const FftPlan& pl,
                            const float2* __restrict__ tw, const float2* __restrict__ roots,
                            int nl, int ls, int es, int tid, int nthr) {
    const float2* s = src;
    float2* d = (src == bufA) ? bufB : bufA;
    for (int st = 0; st < pl.nst; ++st) {
        int R, p, off;
        if (SIGN < 0) { R = pl.rad[st]; p = pl.p_f[st]; off = pl.tw_f[st]; }
        else          { R = pl.rad[pl.nst - 1 - st]; p = pl.p_i[st]; off = pl.tw_i[st]; }
        const int roff = pl.root_off[SIGN < 0 ? st : pl.nst - 1 - st];
        stage_smem<SIGN, LANE_FAST>(s, d, pl.n, R, p, tw + off, roots + roff, nl, ls, es, tid, nthr);
        __syncthreads();
        s = d;
        d = (d == bufA) ? bufB : bufA;
    }
    return const_cast<float2*>(s);
}

}  // namespace oks
