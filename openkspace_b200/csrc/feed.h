// Host-side launch interface of the feeding kernels (k_feed.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace oks {

// One placed acquisition (geometry decided on the host from the headers,
// reader.rs:332-457): samples [src_off, src_off + len) of acquisition `acq`
// go to row (kz, ky), columns [dst_off, dst_off + len), reversed if `reverse`.
struct PlaceEntry {
    long long acq;
    int kz, ky;
    int dst_off, src_off, len;
    int reverse;
    int nc_fit;
};

cudaError_t launch_noise_fit(const float2* noise, int nc, long long ns, double denom, double2* partial_scratch,
                             int max_parts, float2* W, double2* W64, int* status, cudaStream_t st);
// status (nullable): device result word of the noise fit; when it is not 0
// the kernel leaves the data unchanged (no host round trip to decide)
// err (nullable): the context's device error word.  With err given, ns even
// and data on a 16-byte boundary, the bulk-copy staged kernel runs for
// bulk > 0, or for bulk < 0 and nc <= 8; it records 9 in *err if a bounded
// copy wait runs out.
cudaError_t launch_prewhiten_apply(float2* data, const float2* W, long long nacq, int nc, int ns, cudaStream_t st,
                                   const int* status = nullptr, int* err = nullptr, int bulk = -1);
// true when launch_prewhiten_apply takes the bulk-copy kernel for these arguments
bool prewhiten_bulk_eligible(const float2* data, int nc, int ns, const int* err, int bulk);
cudaError_t launch_os_remove(const float2* in, float2* out, long long nlines, const DevPlan& pe, const DevPlan& pr,
                             cudaStream_t st);
cudaError_t launch_place(const float2* src, int nc_src, int ns, const PlaceEntry* tab, long long nent, float2* kspace,
                         int nz, int ny, int nx, cudaStream_t st);

// Navigator phase correction (phasecorr.rs:61-169).  A bin is the
// navigators of one (slice, segment); its scans are entries [first, first +
// count) of the scan list, each [nc][ns] samples at nav + off.
struct PcBin {
    int ns;               // samples per navigator of this bin
    int first, count;
    int pad;
    long long corr;       // offset of the bin's correction vector (ns entries)
};
struct PcScan {
    long long off;
    int nc, pad;
};
// c(k) = conj(avg_k) / |avg_k| of the coil-summed navigators of each bin
cudaError_t launch_phasecorr_fit(const float2* nav, const PcScan* scans, const PcBin* bins, int nbins, int max_ns,
                                 float2* corr, cudaStream_t st);
// data[a][c][k] *= c_bin(a)(k) for k < min(ns, bin ns); scan_bin[a] < 0: untouched
cudaError_t launch_phasecorr_apply(float2* data, long long nacq, int nc, int ns, const int* scan_bin,
                                   const PcBin* bins, const float2* corr, cudaStream_t st);

}  // namespace oks
