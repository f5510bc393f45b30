/*
 * okscuda.h -- C-ABI of the B200 (sm_100a) FISTA-CS path of OpenKSpace.
 *
 * Plain C: pointers, sizes and int status codes.  No C++ types cross the
 * boundary and nothing throws.  Reference paths are relative to the
 * OpenKSpace project (crates/...).
 *
 * Conventions
 *  - Complex data is interleaved (re, im) float32 pairs: okscuda_c64, the
 *    layout of the reference's num_complex::Complex32.
 *  - Arrays are C-order.  Pointers named d_* are device pointers (from
 *    okscuda_malloc or any CUDA allocation on the context's device);
 *    pointers named h_* are host pointers.
 *  - Compute entry points are asynchronous on the context's stream
 *    (okscuda_set_stream); okscuda_download / okscuda_synchronize wait.
 *  - Return 0 (OKS_OK) on success or a negative OKS_E* code; the message is
 *    kept in the context (okscuda_last_error).
 *  - A context is bound to one device and is not thread-safe: one context
 *    per host thread, as the reference's strategy is called from one thread.
 */
#ifndef OKSCUDA_H
#define OKSCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } okscuda_c64;
typedef struct okscuda_ctx okscuda_ctx;

enum {
    OKS_OK = 0,
    OKS_EINVAL = -1,     /* bad argument (null pointer, negative size, ...)            */
    OKS_ESHAPE = -2,     /* shapes disagree (cs.rs:43-47 CsError::ShapeMismatch)        */
    OKS_EODD = -3,       /* odd ny or nx (cs.rs:49-50 CsError::OddDimension)            */
    OKS_ENOTPD = -4,     /* noise covariance not positive definite (prewhiten.rs:161)   */
    OKS_ECUDA = -5,      /* CUDA runtime error                                          */
    OKS_ENOMEM = -6,     /* device allocation failed                                    */
    OKS_EAGAIN = -7,     /* admission refused, retry later                              */
    OKS_ETIMEDOUT = -8,  /* a bounded wait ran out                                      */
    OKS_ENOTSUP = -9,    /* size or mode outside what this build supports               */
    OKS_ESKIP = -10      /* the reference would silently skip this step (returns None)  */
};

/* ---------------------------------------------------------------- context */
int okscuda_create(int device, okscuda_ctx** out);
void okscuda_destroy(okscuda_ctx* ctx);
/* Copies the last error message (NUL-terminated, truncated to len). */
int okscuda_last_error(const okscuda_ctx* ctx, char* buf, size_t len);
/* Use an existing cudaStream_t (passed as void*); NULL restores the
 * context's own stream. */
int okscuda_set_stream(okscuda_ctx* ctx, void* stream);
void* okscuda_get_stream(okscuda_ctx* ctx);
int okscuda_synchronize(okscuda_ctx* ctx);
const char* okscuda_version(void);

/* ---------------------------------------------------------- device memory */
int okscuda_malloc(okscuda_ctx* ctx, size_t bytes, void** d_ptr);
int okscuda_free(okscuda_ctx* ctx, void* d_ptr);
/* Host<->device copies on the context stream; download waits for completion. */
int okscuda_upload(okscuda_ctx* ctx, void* d_dst, const void* h_src, size_t bytes);
int okscuda_download(okscuda_ctx* ctx, void* h_dst, const void* d_src, size_t bytes);
int okscuda_host_alloc(okscuda_ctx* ctx, size_t bytes, void** h_ptr);   /* pinned */
int okscuda_host_free(okscuda_ctx* ctx, void* h_ptr);

/* ------------------------------------------------------------- primitives */
/* cs.rs:141-178 centred_fft2 / cs.rs:180-218 centred_ifft2 on batch x [ny, nx],
 * in place: ifftshift -> DFT rows -> DFT columns -> fftshift -> 1/sqrt(ny nx). */
int okscuda_centred_fft2(okscuda_ctx* ctx, okscuda_c64* d_data, int batch, int ny, int nx,
                         int inverse);
/* wavelet.rs:32-52 haar_forward / wavelet.rs:55-75 haar_inverse, batch x [ny, nx]. */
int okscuda_haar_forward(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, int batch,
                         int ny, int nx);
int okscuda_haar_inverse(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, int batch,
                         int ny, int nx);
/* wavelet.rs:80-99 soft_threshold_details, in place. */
int okscuda_soft_threshold_details(okscuda_ctx* ctx, okscuda_c64* d_data, int batch, int ny, int nx,
                                   float lambda);
/* coil.rs:24-27 / strategy.rs:870-879 RSS over nc coils of [ny, nx], then the
 * centre crop of crop.rs:13-27 to [ty, tx] (ty = ny, tx = nx for no crop). */
int okscuda_rss_crop(okscuda_ctx* ctx, const okscuda_c64* d_coils, int nc, int ny, int nx, int ty,
                     int tx, float* d_out);

/* ---------------------------------------------------------------- FISTA-CS */
/* cs.rs:59-139 fista_cs_single_coil, batched: `batch` independent problems
 * d_kspace[batch, ny, nx] sharing the host mask h_mask[ny, nx] (0/1 bytes).
 * Result d_out[batch, ny, nx]; d_out may equal d_kspace.  Errors: OKS_EODD
 * for odd ny/nx (cs.rs:72-74). */
int okscuda_fista_cs(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int batch,
                     int ny, int nx, int iters, float lambda, okscuda_c64* d_out);

/* strategy.rs:850-880, one kz slice: per-coil FISTA on d_kspace[nc, ny, nx]
 * with the slice mask h_mask[ny, nx], then f32 RSS in coil order into
 * d_rss[ny, nx].  d_coils[nc, ny, nx] receives the coil images when not NULL. */
int okscuda_cs_slice(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc,
                     int ny, int nx, int iters, float lambda, float* d_rss, okscuda_c64* d_coils);

#ifdef __cplusplus
}
#endif
#endif /* OKSCUDA_H */
