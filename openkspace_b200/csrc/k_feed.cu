// sm_100a kernels that feed the FISTA-CS loop (the reference's read closure,
// strategy.rs:807-815, and its calibration, strategy.rs:783-798):
//   prewhiten.rs:48-111   noise covariance Psi           -> k_noise_cov (FP64, chunked, ordered sum)
//   prewhiten.rs:148-210  Cholesky L, W = L^-1            -> k_chol_inv (FP64, one CTA)
//   prewhiten.rs:118-142  s <- W s per sample column       -> k_prewhiten_apply
//   oversampling.rs:103-155 centred IFFT/crop/FFT          -> k_os_remove
//   reader.rs:332-457     line placement (first-wins, reverse, centring decided on the host)
//                                                          -> k_place
//   phasecorr.rs:61-169   navigator correction vectors / per-line phasor
//                                                          -> k_phasecorr_fit, k_phasecorr_apply
#include <cuda_runtime.h>
#include <float.h>

#include "fft_dev.cuh"
#include "feed.h"

namespace oks {

// -------------------------------------------------------- noise covariance
// Lower triangle (incl. diagonal) of sum_n s(n) s(n)^H over samples
// [n0, n0 + chunk) of noise[nc][ns]; partial sums in FP64, one per CTA.
__global__ void k_noise_cov(const float2* __restrict__ noise, int nc, long long ns, long long chunk,
                            double2* __restrict__ partial) {
    const long long n0 = blockIdx.x * chunk;
    const long long n1 = min(ns, n0 + chunk);
    const int npair = nc * (nc + 1) / 2;
    double2* out = partial + (size_t)blockIdx.x * npair;
    for (int q = threadIdx.x; q < npair; q += blockDim.x) {
        // q -> (j, i) with j >= i : row-major lower triangle
        int j = (int)((sqrt(8.0 * q + 1.0) - 1.0) / 2.0);
        while ((j + 1) * (j + 2) / 2 <= q) ++j;
        while (j * (j + 1) / 2 > q) --j;
        const int i = q - j * (j + 1) / 2;
        double re = 0.0, im = 0.0;
        const float2* sj = noise + (long long)j * ns;
        const float2* si = noise + (long long)i * ns;
        for (long long n = n0; n < n1; ++n) {
            const float2 a = sj[n], b = si[n];
            // psi[j][i] += s_j * conj(s_i)      (prewhiten.rs:89-93)
            re += (double)a.x * b.x + (double)a.y * b.y;
            im += (double)a.y * b.x - (double)a.x * b.y;
        }
        out[q] = make_double2(re, im);
    }
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {   // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Sums the partials in chunk order, scales by 1/max(total-1, 1), then
// Cholesky (prewhiten.rs:148-179) and the triangular inverse
// (prewhiten.rs:183-210), all in FP64.  status: 0 ok, 1 not positive
// definite, 2 singular diagonal.  W (complex64, [nc][nc], upper zero) and
// W64 (FP64) are written only when status == 0.
__global__ void k_chol_inv(const double2* __restrict__ partial, int nparts, int nc, double denom,
                           float2* __restrict__ W, double2* __restrict__ W64, int* __restrict__ status) {
    extern __shared__ double2 zs[];
    double2* A = zs;              // Psi   [nc][nc]
    double2* L = A + nc * nc;     // L     [nc][nc]
    double2* V = L + nc * nc;     // L^-1  [nc][nc]
    __shared__ int bad;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int npair = nc * (nc + 1) / 2;
    if (tid == 0) bad = 0;
    for (int q = tid; q < nc * nc; q += nthr) {
        A[q] = make_double2(0.0, 0.0);
        L[q] = make_double2(0.0, 0.0);
        V[q] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int q = tid; q < npair; q += nthr) {
        int j = 0;
        while ((j + 1) * (j + 2) / 2 <= q) ++j;
        const int i = q - j * (j + 1) / 2;
        double re = 0.0, im = 0.0;
        for (int b = 0; b < nparts; ++b) {
            re += partial[(size_t)b * npair + q].x;
            im += partial[(size_t)b * npair + q].y;
        }
        A[j * nc + i] = make_double2(re / denom, im / denom);
    }
    __syncthreads();
    for (int i = 0; i < nc; ++i) {
        if (tid == 0) {
            double2 d = A[i * nc + i];
            for (int k = 0; k < i; ++k) {
                const double2 t = zmulc(L[i * nc + k], L[i * nc + k]);
                d.x -= t.x;
                d.y -= t.y;
            }
            if (!(isfinite(d.x)) || d.x <= 0.0) bad = 1;
            else L[i * nc + i] = make_double2(sqrt(d.x), 0.0);
        }
        __syncthreads();
        if (bad) break;
        const double inv = 1.0 / L[i * nc + i].x;
        for (int j = i + 1 + tid; j < nc; j += nthr) {
            double2 s = A[j * nc + i];
            for (int k = 0; k < i; ++k) {
                const double2 t = zmulc(L[j * nc + k], L[i * nc + k]);
                s.x -= t.x;
                s.y -= t.y;
            }
            L[j * nc + i] = make_double2(s.x * inv, s.y * inv);
        }
        __syncthreads();
    }
    if (bad) {
        if (tid == 0) *status = 1;
        return;
    }
    // forward substitution per unit column, one column per thread
    for (int col = tid; col < nc; col += nthr) {
        for (int i = 0; i < nc; ++i) {
            double2 s = make_double2(i == col ? 1.0 : 0.0, 0.0);
            for (int j = 0; j < i; ++j) {
                const double2 t = zmul(L[i * nc + j], V[j * nc + col]);
                s.x -= t.x;
                s.y -= t.y;
            }
            const double2 d = L[i * nc + i];
            if (fabs(d.x) < (double)FLT_EPSILON && fabs(d.y) < (double)FLT_EPSILON) {
                atomicExch(&bad, 2);
                break;
            }
            const double den = d.x * d.x + d.y * d.y;
            V[i * nc + col] = make_double2((s.x * d.x + s.y * d.y) / den, (s.y * d.x - s.x * d.y) / den);
        }
    }
    __syncthreads();
    if (bad) {
        if (tid == 0) *status = 2;
        return;
    }
    for (int q = tid; q < nc * nc; q += nthr) {
        const int i = q / nc, j = q - i * nc;
        const double2 v = (j <= i) ? V[q] : make_double2(0.0, 0.0);
        W[q] = make_float2((float)v.x, (float)v.y);
        if (W64) W64[q] = v;
    }
    if (tid == 0) *status = 0;
}

// ------------------------------------------------------- prewhiten apply
// data [nacq][nc][ns]: every sample column s -> W s (lower triangular).
// One column through W, with its nc samples in registers: out_i =
// sum_{j <= i} W_ij s_j in j order (prewhiten.rs:126-135).  Both apply
// kernels call this, so they round identically.
template <int NCMAX, class LD, class ST>
__device__ __forceinline__ void whiten_column(const float2* __restrict__ W, int wstride, int nc, LD ld, ST st) {
    float2 s[NCMAX];
#pragma unroll
    for (int j = 0; j < NCMAX; ++j) s[j] = (j < nc) ? ld(j) : make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < NCMAX; ++i) {
        if (i >= nc) break;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j <= i; ++j) acc = acc + cmul(W[i * wstride + j], s[j]);
        st(i, acc);
    }
}

template <int NCMAX>
__global__ void k_prewhiten_apply(float2* __restrict__ data, const float2* __restrict__ Wg, long long nacq, int nc,
                                  int ns, const int* __restrict__ status) {
    // status (optional): the noise fit's result word; anything but 0 means
    // the fit returned None (prewhiten.rs:161) and the data stay as they are
    if (status && *status != 0) return;
    __shared__ float2 W[NCMAX * NCMAX];
    for (int q = threadIdx.x; q < nc * nc; q += blockDim.x) W[(q / nc) * NCMAX + q % nc] = Wg[q];
    __syncthreads();
    const long long total = nacq * ns;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long a = t / ns;
        const int n = (int)(t - a * ns);
        float2* col = data + a * nc * (long long)ns + n;
        whiten_column<NCMAX>(
            W, NCMAX, nc, [&](int j) { return col[(long long)j * ns]; },
            [&](int i, float2 v) { col[(long long)i * ns] = v; });
    }
}

// Bulk-copy staged prewhitening.  A CTA of TS threads loops over tiles of
// (acquisition a, samples [s0, s0 + TS)).  Lane c < nc of warp 0 copies
// channel c's row segment (8 len contiguous bytes) into a shared stage with
// cp.async.bulk, completing on the stage's mbarrier; with two stages the next
// tile's copies are in flight while this one is computed, and they cost no
// issue slots or registers.  Thread s reads its sample column from the stage,
// applies W (whiten_column) and stores the results straight to global memory
// (consecutive threads, consecutive samples of a channel row); the barrier at
// the end of the tile frees the stage for the copies issued one tile later.
// (Staging the results for bulk stores as well measured slower on B200: the
// refill of a stage then waits for its stores to have been read.)
// The launcher takes this kernel only for ns even and a 16-byte aligned data
// pointer: every segment then starts on a 16-byte boundary and is a multiple
// of 16 bytes long.  Each mbarrier wait is bounded (about one second of clock
// cycles); on time-out the CTA records 9 in *err, waits (bounded again) for
// its loads in flight and returns.
__device__ __forceinline__ uint32_t pw_smem(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool pw_try(uint32_t bar, uint32_t parity) {
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
__device__ __forceinline__ bool pw_wait(uint32_t bar, uint32_t parity) {
    constexpr long long kCycles = 2000000000ll;   // about one second at 1.9 GHz
    if (pw_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!pw_try(bar, parity))
        if (clock64() - t0 > kCycles) return false;
    return true;
}

template <int NCMAX, int TS>
__global__ void __launch_bounds__(TS) k_prewhiten_bulk(float2* __restrict__ data, const float2* __restrict__ Wg,
                                                       long long nacq, int nc, int ns, const int* __restrict__ status,
                                                       int* __restrict__ err) {
    if (status && *status != 0) return;
    extern __shared__ __align__(16) float2 pw_sm[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(pw_sm);   // two stage barriers (16 bytes)
    float2* W = pw_sm + 2;                                 // [nc][nc]
    float2* stg0 = W + ((nc * nc + 1) & ~1);               // two stages [nc][TS], 16-byte aligned
    const int tid = threadIdx.x;
    const bool issuer = tid < nc;                          // nc <= 32: lanes of warp 0
    for (int q = tid; q < nc * nc; q += TS) W[q] = Wg[q];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pw_smem(&bars[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pw_smem(&bars[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const long long tiles_per = (ns + TS - 1) / TS;
    const long long total = nacq * tiles_per;
    // tile u -> (acquisition, first sample, length); the caller of issue is lane c
    auto tile_of = [&](long long u, long long& a, int& s0, int& len) {
        a = u / tiles_per;
        s0 = (int)(u - a * tiles_per) * TS;
        len = min(TS, ns - s0);
    };
    auto issue_load = [&](long long u, int b) {   // warp 0 only
        long long a;
        int s0, len;
        tile_of(u, a, s0, len);
        const uint32_t bar = pw_smem(&bars[b]);
        if (tid == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"((uint32_t)(nc * len * 8))
                         : "memory");
        __syncwarp();
        if (issuer) {
            const float2* src = data + (a * nc + tid) * (long long)ns + s0;
            float2* dst = stg0 + ((size_t)b * nc + tid) * TS;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             pw_smem(dst)),
                         "l"(src), "r"((uint32_t)(len * 8)), "r"(bar)
                         : "memory");
        }
    };
    long long u = blockIdx.x;
    if (tid < 32 && u < total) issue_load(u, 0);
    uint32_t use0 = 0u, use1 = 0u;   // completed waits per stage: the parity of its next phase
    int it = 0;
    for (; u < total; u += gridDim.x, ++it) {
        const int b = it & 1;
        const long long un = u + gridDim.x;
        const bool pending_next = un < total;
        if (tid < 32 && pending_next) issue_load(un, b ^ 1);
        const uint32_t par = (b ? use1 : use0) & 1u, par_next = (b ? use0 : use1) & 1u;
        const bool ok = pw_wait(pw_smem(&bars[b]), par);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(err, 9);
                pw_wait(pw_smem(&bars[b]), par);                       // copies in flight land first
                if (pending_next) pw_wait(pw_smem(&bars[b ^ 1]), par_next);
            }
            break;
        }
        if (b) ++use1;
        else ++use0;
        long long a;
        int s0, len;
        tile_of(u, a, s0, len);
        const float2* stg = stg0 + (size_t)b * nc * TS;
        float2* out = data + a * nc * (long long)ns + s0 + tid;
        if (tid < len)
            whiten_column<NCMAX>(
                W, nc, nc, [&](int j) { return stg[j * TS + tid]; },
                [&](int i, float2 v) { out[(long long)i * ns] = v; });
        __syncthreads();                                   // stage b read by every thread: free for a refill
    }
}

bool prewhiten_bulk_eligible(const float2* data, int nc, int ns, const int* err, int bulk) {
    // bulk < 0 (the default): by channel count, the bulk copies for nc <= 8,
    // where they measured faster on B200 than the plain loads (at 15 and 32
    // channels the plain kernel was faster)
    return (bulk > 0 || (bulk < 0 && nc <= 8)) && err && nc >= 1 && nc <= 32 && ns > 0 && (ns % 2) == 0 &&
           (reinterpret_cast<uintptr_t>(data) % 16) == 0;
}

template <int NCMAX, int TS>
static cudaError_t launch_bulk(float2* data, const float2* W, long long nacq, int nc, int ns, cudaStream_t st,
                               const int* status, int* err) {
    const size_t smem = 16 + sizeof(float2) * (size_t)(((nc * nc + 1) & ~1) + 2 * nc * TS);
    cudaError_t e =
        cudaFuncSetAttribute(k_prewhiten_bulk<NCMAX, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prewhiten_bulk<NCMAX, TS>, TS, smem);
    const long long tiles = nacq * ((ns + TS - 1) / TS);
    long long blocks = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (blocks > tiles) blocks = tiles;
    k_prewhiten_bulk<NCMAX, TS><<<(unsigned)blocks, TS, smem, st>>>(data, W, nacq, nc, ns, status, err);
    return cudaGetLastError();
}

cudaError_t launch_prewhiten_apply(float2* data, const float2* W, long long nacq, int nc, int ns, cudaStream_t st,
                                   const int* status, int* err, int bulk) {
    const long long total = nacq * ns;
    if (total <= 0 || nc <= 0) return cudaSuccess;
    if (prewhiten_bulk_eligible(data, nc, ns, err, bulk)) {
        if (nc <= 8) return launch_bulk<8, 128>(data, W, nacq, nc, ns, st, status, err);
        if (nc <= 16) return launch_bulk<16, 128>(data, W, nacq, nc, ns, st, status, err);
        return launch_bulk<32, 128>(data, W, nacq, nc, ns, st, status, err);
    }
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (nc <= 8) k_prewhiten_apply<8><<<(unsigned)blocks, 256, 0, st>>>(data, W, nacq, nc, ns, status);
    else if (nc <= 16) k_prewhiten_apply<16><<<(unsigned)blocks, 256, 0, st>>>(data, W, nacq, nc, ns, status);
    else if (nc <= 32) k_prewhiten_apply<32><<<(unsigned)blocks, 256, 0, st>>>(data, W, nacq, nc, ns, status);
    else if (nc <= 64) k_prewhiten_apply<64><<<(unsigned)blocks, 128, 0, st>>>(data, W, nacq, nc, ns, status);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ------------------------------------------------- navigator phase correction
// One thread per (bin, sample k), in the reference's FP32 order: each
// navigator's coil sum sum_c s_c(k) (channels in order), added to the bin in
// scan order (phasecorr.rs:76-102); then avg = sum * (1 / count) and
// c(k) = conj(avg) / |avg| with num_complex's division by (|avg|, 0), or 1
// where |avg| < 1e-20 (phasecorr.rs:106-119).
__global__ void k_phasecorr_fit(const float2* __restrict__ nav, const PcScan* __restrict__ scans,
                                const PcBin* __restrict__ bins, float2* __restrict__ corr) {
    const PcBin b = bins[blockIdx.y];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < b.ns; k += gridDim.x * blockDim.x) {
        float sr = 0.f, si = 0.f;
        for (int q = b.first; q < b.first + b.count; ++q) {
            const PcScan sc = scans[q];
            float cr = 0.f, ci = 0.f;
            for (int c = 0; c < sc.nc; ++c) {
                const float2 v = nav[sc.off + (long long)c * b.ns + k];
                cr = __fadd_rn(cr, v.x);
                ci = __fadd_rn(ci, v.y);
            }
            sr = __fadd_rn(sr, cr);
            si = __fadd_rn(si, ci);
        }
        const float inv_n = __fdiv_rn(1.f, (float)b.count);
        const float ar = __fmul_rn(sr, inv_n), ai = __fmul_rn(si, inv_n);
        const float mag = hypotf(ar, ai);
        float2 out = make_float2(1.f, 0.f);
        if (!(mag < 1e-20f)) {
            const float n2 = __fmul_rn(mag, mag);
            out = make_float2(__fdiv_rn(__fmul_rn(ar, mag), n2), __fdiv_rn(__fmul_rn(-ai, mag), n2));
        }
        corr[b.corr + k] = out;
    }
}

// row[k] *= c(k), k < min(ns, len(c)), every channel (phasecorr.rs:141-168)
__global__ void k_phasecorr_apply(float2* __restrict__ data, long long nacq, int nc, int ns,
                                  const int* __restrict__ scan_bin, const PcBin* __restrict__ bins,
                                  const float2* __restrict__ corr) {
    const long long per = (long long)nc * ns, total = nacq * per;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long a = t / per;
        const int k = (int)((t - a * per) % ns);
        const int b = scan_bin[a];
        if (b < 0) continue;
        const PcBin bb = bins[b];
        if (k >= min(ns, bb.ns)) continue;
        data[t] = cmul(data[t], corr[bb.corr + k]);
    }
}

cudaError_t launch_phasecorr_fit(const float2* nav, const PcScan* scans, const PcBin* bins, int nbins, int max_ns,
                                 float2* corr, cudaStream_t st) {
    if (nbins <= 0 || max_ns <= 0) return cudaSuccess;
    if (nbins > 65535) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((max_ns + 127) / 128), (unsigned)nbins);
    k_phasecorr_fit<<<grid, 128, 0, st>>>(nav, scans, bins, corr);
    return cudaGetLastError();
}

cudaError_t launch_phasecorr_apply(float2* data, long long nacq, int nc, int ns, const int* scan_bin,
                                   const PcBin* bins, const float2* corr, cudaStream_t st) {
    const long long total = nacq * nc * (long long)ns;
    if (total <= 0) return cudaSuccess;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_phasecorr_apply<<<(unsigned)blocks, 256, 0, st>>>(data, nacq, nc, ns, scan_bin, bins, corr);
    return cudaGetLastError();
}

cudaError_t launch_noise_fit(const float2* noise, int nc, long long ns, double denom, double2* partial_scratch,
                             int max_parts, float2* W, double2* W64, int* status, cudaStream_t st) {
    if (nc <= 0 || nc > 128) return cudaErrorInvalidValue;
    long long chunk = 4096;
    long long parts = (ns + chunk - 1) / chunk;
    if (parts > max_parts) {
        chunk = (ns + max_parts - 1) / max_parts;
        parts = (ns + chunk - 1) / chunk;
    }
    if (parts < 1) parts = 1;
    k_noise_cov<<<(unsigned)parts, 256, 0, st>>>(noise, nc, ns, chunk, partial_scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t smem = sizeof(double2) * 3 * (size_t)nc * nc;
    e = cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_chol_inv<<<1, 128, smem, st>>>(partial_scratch, (int)parts, nc, denom, W, W64, status);
    return cudaGetLastError();
}

// -------------------------------------------------- oversampling removal
// in [nlines][enc] -> out [nlines][rec]: ifftshift, IDFT, *1/enc, fftshift,
// crop [(enc-rec)/2, +rec), ifftshift, DFT, fftshift (oversampling.rs:122-145).
__global__ void k_os_remove(const float2* __restrict__ in, float2* __restrict__ out, long long nlines, int enc,
                            int rec, FftPlan pe, const float2* __restrict__ twe, const float2* __restrict__ rte,
                            int rte_n, FftPlan pr, const float2* __restrict__ twr, const float2* __restrict__ rtr,
                            int rtr_n, int lpc) {
    extern __shared__ float2 sm[];
    float2* A = sm;
    float2* B = A + (size_t)lpc * enc;
    float2* TWE = B + (size_t)lpc * enc;
    float2* RTE = TWE + pe.tw_total;
    float2* TWR = RTE + rte_n;
    float2* RTR = TWR + pr.tw_total;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int q = tid; q < pe.tw_total; q += nthr) TWE[q] = twe[q];
    for (int q = tid; q < rte_n; q += nthr) RTE[q] = rte[q];
    for (int q = tid; q < pr.tw_total; q += nthr) TWR[q] = twr[q];
    for (int q = tid; q < rtr_n; q += nthr) RTR[q] = rtr[q];
    const long long l0 = (long long)blockIdx.x * lpc;
    const int c1 = (enc + 1) / 2;
    for (int q = tid; q < lpc * enc; q += nthr) {
        const int l = q / enc, m = q - l * enc;
        int src = m + c1;
        if (src >= enc) src -= enc;
        A[q] = (l0 + l < nlines) ? in[(l0 + l) * enc + src] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* X = fft_smem<+1, false>(A, A, B, pe, TWE, RTE, lpc, enc, 1, tid, nthr);
    float2* C = (X == A) ? B : A;
    // cropped[i] = fftshift(X)[start + i] = X[(start + i + enc/2) % enc];
    // then the rec-point ifftshift: buf[m] = cropped[(m + ceil(rec/2)) % rec]
    const int start = (enc - rec) / 2, h = enc / 2, cr = (rec + 1) / 2;
    const float sc = 1.0f / (float)enc;
    for (int q = tid; q < lpc * rec; q += nthr) {
        const int l = q / rec, m = q - l * rec;
        int i = m + cr;
        if (i >= rec) i -= rec;
        int k = start + i + h;
        if (k >= enc) k -= enc;
        C[l * rec + m] = X[l * enc + k] * sc;
    }
    __syncthreads();
    float2* Y = fft_smem<-1, false>(C, C, X, pr, TWR, RTR, lpc, rec, 1, tid, nthr);
    const int h2 = rec / 2;
    for (int q = tid; q < lpc * rec; q += nthr) {
        const int l = q / rec, k = q - l * rec;
        if (l0 + l >= nlines) continue;
        int src = k + h2;
        if (src >= rec) src -= rec;
        out[(l0 + l) * rec + k] = Y[l * rec + src];
    }
}

cudaError_t launch_os_remove(const float2* in, float2* out, long long nlines, const DevPlan& pe, const DevPlan& pr,
                             cudaStream_t st) {
    const int enc = pe.plan.n, rec = pr.plan.n;
    if (nlines <= 0) return cudaSuccess;
    int lpc = 8192 / enc;
    if (lpc < 1) lpc = 1;
    if (lpc > 16) lpc = 16;
    size_t smem = sizeof(float2) * ((size_t)2 * lpc * enc + pe.plan.tw_total + pe.roots_total + pr.plan.tw_total +
                                    pr.roots_total);
    cudaError_t e = cudaFuncSetAttribute(k_os_remove, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    long long grid = (nlines + lpc - 1) / lpc;
    k_os_remove<<<(unsigned)grid, 256, smem, st>>>(in, out, nlines, enc, rec, pe.plan, pe.tw, pe.roots, pe.roots_total,
                                                   pr.plan, pr.tw, pr.roots, pr.roots_total, lpc);
    return cudaGetLastError();
}

// ------------------------------------------------------------- placement
// One placed acquisition per CTA row: kspace[c][kz][ky][dst + i] =
// src[a][c][src_off + (reverse ? len-1-i : i)] for c < nc_fit, i < len.
__global__ void k_place(const float2* __restrict__ src, int nc_src, int ns, const PlaceEntry* __restrict__ tab,
                        long long nent, float2* __restrict__ kspace, int nz, int ny, int nx) {
    for (long long e = blockIdx.x; e < nent; e += gridDim.x) {
        const PlaceEntry t = tab[e];
        const float2* s = src + t.acq * (long long)nc_src * ns;
        for (int q = threadIdx.x; q < t.nc_fit * t.len; q += blockDim.x) {
            const int c = q / t.len, i = q - c * t.len;
            const int si = t.src_off + (t.reverse ? t.len - 1 - i : i);
            kspace[(((long long)c * nz + t.kz) * ny + t.ky) * nx + t.dst_off + i] = s[(long long)c * ns + si];
        }
    }
}

cudaError_t launch_place(const float2* src, int nc_src, int ns, const PlaceEntry* tab, long long nent, float2* kspace,
                         int nz, int ny, int nx, cudaStream_t st) {
    if (nent <= 0) return cudaSuccess;
    long long blocks = nent < 148 * 16 ? nent : 148 * 16;
    k_place<<<(unsigned)blocks, 256, 0, st>>>(src, nc_src, ns, tab, nent, kspace, nz, ny, nx);
    return cudaGetLastError();
}

}  // namespace oks
