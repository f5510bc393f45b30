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
/* Tuning knobs (no reference counterpart):
 *   "col_engine"    ky-only masks: 0 auto (register-resident kernel where a
 *                   compile-time plan exists for ny), 1 generic shared-memory
 *                   kernel, 2 register kernel (falls back to 1 for other ny)
 *   "col_variant"   register column engine: -1 (default) per column length
 *                   (the E = 8 alternative for 256, 320, 384, 512), 0 primary
 *                   plan, 1 the E = 8 alternative where one exists (192, 256,
 *                   320, 384, 512)
 *   "fista2d_chunk" problems per chunk of the 2-D-mask engine (0 = auto,
 *                   sized for L2 residency)
 *   "row_engine"    2-D-mask engine, readout-direction transforms: 0 (default)
 *                   SIMT FFT fused with the prox; 1 tensor-core DFT-as-GEMM
 *                   (split 3xBF16, okscuda_dft_rows engine 1) over the sampled
 *                   kx columns, with the prox in between (nx <= 2048)
 *   "tc_gate_test"  tests of the bounded waits only: > 0 makes every
 *                   tensor-core launch of okscuda_dft_rows first wait at most
 *                   that many clock cycles on a device word nothing sets; it
 *                   then records code 7 (okscuda_tc_status) and returns with
 *                   no work issued.  0 (default) off
 *   "fista2d_streams" chunks of the 2-D-mask engine in flight at once, on
 *                   forked streams with separate state (1 to 8, default 2)
 *   "persist2d"     2-D register passes: 1 (default) = one CTA per resident
 *                   slot, units grid-strided; 0 = one CTA per unit
 *   "mask_bits"     2-D column pass: 1 = separable masks are read as row
 *                   and column bits instead of mask bytes
 *   "prefetch2d"    2-D register passes, the next unit's loads issued
 *                   (cp.async) before the current unit's transforms: bit 0
 *                   column pass with separable masks (default 1), bit 1 row
 *                   pass; bit 2 row pass with the next row pair of S, Z~ and
 *                   X~ staged in shared memory by cp.async.bulk (mbarrier
 *                   completion, bounded waits)
 *   "col2d_lanes"   2-D-mask engine column pass: 0 (default) by length (form 14
 *                   at ny = 368, else -1); -1 one column pair
 *                   per thread group; 1-8 the lanes form (tiles of 8 or 16
 *                   columns in shared memory, lanes across the columns; the
 *                   forms of "xform_lanes", 5-8 for 368); 9-12 for ny = 368
 *                   and separable masks, the lanes form pruned to the
 *                   sampled rows (radix-23 output pairs and input pairs that
 *                   only unsampled rows reach are left out), (columns,
 *                   threads per column) (8,16) (8,32) (16,16) (16,32); 13 =
 *                   (8,16) with the row slots swizzled against bank conflicts;
 *                   14 = the two-stage plan 16 · 23 with the residual fused
 *                   between the directions in registers
 *   "pdl2d"         2-D register passes launched as programmatic dependent
 *                   launches: a pass's CTAs load their tables while the
 *                   previous pass ends, then wait for it (griddepcontrol);
 *                   0 (default) plain stream order, 1 on
 *   "row2d_ctas", "col2d_ctas" 2-D engine: at most this many CTAs per SM for
 *                   the persistent row pass / the pruned 368 column pass, so
 *                   the other stream's pass finds room on every SM; 0
 *                   (default) = every resident slot
 *   "occ2d"         2-D register passes: 1 = launch bounds that keep at
 *                   least 12 warps resident per SM, 2 = at least 18, 3 = at
 *                   least 15, 0 = registers as needed
 *   "autotune_use"  1 (default): shapes in the autotune table use their
 *                   tuned choices in place of the options above; 0: ignore
 *                   the table
 *   "autotune_clear" (any value) empties the autotune table
 *   "xform_engine"  centred row / column transforms (okscuda_centred_fft2,
 *                   okscuda_ifft2, okscuda_ifft1_kz, okscuda_dft_rows engine 0
 *                   and the column engine's readout pass): 1 (default)
 *                   register-resident kernels for the lengths with a compile-
 *                   time plan (128, 192, 256, 320, 368, 384, 512, 640), 0 the
 *                   shared-memory mixed-radix kernels for every length
 *   "xform_tile"    register column transform: column pairs per CTA, 0
 *                   (default: 8, or 4 where 8 do not fit), 2, 4 or 8
 *   "xform_lanes"   register column transform with the lanes across the
 *                   columns (whole row segments straight from and to global
 *                   memory): 0 (default) for the lengths where it is faster
 *                   (192, 256, 320, 368, 384, 512, 640), 1-4 a (columns, threads per column)
 *                   form (16,32) (16,64) (8,64) (8,32) for every length but 368,
 *                   5-8 the 368 forms (16,16) (8,16) (16,32) (8,32), 16
 *                   threads per column being one per radix-23 butterfly,
 *                   9 the two-stage 368 form (16 · 23, 8 columns, the default),
 *                   10 the two-stage 640 form (20 · 32, 8 columns, the default),
 *                   11 the two-stage 320 form (16 · 20, 8 columns, the default),
 *                   -1 never
 *   "xform_row_variant" register row transform: 0 (default) the fastest plan
 *                   per length; 1 the E = 8 plans for 192 (8·3·8) and 320
 *                   (8·5·8); 2 the 96-thread plan 4·12·4 for 192 (measurement);
 *                   3 the two-stage forms at 368 (16 · 23) and 320 (16 · 20),
 *                   8 rows per CTA, rows on 16-byte boundaries (also the
 *                   default at those lengths)
 *   "xform_lanes_pf" lanes form: 1 (default) = software-pipelined (the next
 *                   tile is copied into shared memory with cp.async while the
 *                   current one is transformed; even nx and 16-byte aligned
 *                   data), 0 = stage 0 reads global memory directly
 *   "prewhiten_bulk" prewhitening: 1 = tiles of 128 samples of every
 *                   channel staged in shared memory by bulk copies
 *                   (cp.async.bulk, two stages) for nc <= 32, even ns and
 *                   16-byte aligned data, a time-out of its bounded copy
 *                   waits reported as 9 by okscuda_tc_status; 0 = plain
 *                   loads; -1 (default) = the bulk copies for nc <= 8, plain
 *                   loads above (the faster of the two on B200)
 * Any other name returns OKS_EINVAL. */
int okscuda_set_option(okscuda_ctx* ctx, const char* name, long long value);
/* Autotuner (no reference counterpart): times the plan and launch-shape
 * candidates of the FISTA engine for one shape on seeded synthetic data on
 * the device and keeps the fastest for that shape in the context's table.
 * kind 0: ky-only masks (column engine: register plan variants, generic
 * kernel; the choice applies to every nx).  kind 1: 2-D masks with partial
 * rows (register budget, pipelined loads, chunks in flight, chunk size).  nc
 * problems, `iters` iterations per timing call.  A JSON report of every
 * candidate's time and the choice is written to report (may be NULL). */
int okscuda_autotune(okscuda_ctx* ctx, int kind, int ny, int nx, int nc, int iters, char* report,
                     size_t report_len);
/* The table as text, one line per shape ("kind ny nx col_engine col_variant
 * persist2d occ2d prefetch2d fista2d_streams fista2d_chunk"), and loading such
 * text back (added to the table; OKS_EINVAL on a malformed line). */
int okscuda_autotune_table(okscuda_ctx* ctx, char* buf, size_t len);
int okscuda_autotune_load(okscuda_ctx* ctx, const char* text);

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
/* The row (readout-direction) pass of cs.rs:141-178: nrows rows of length n,
 * each transformed by an unnormalised DFT (inverse = 1: e^{+}), with the
 * ifftshift/fftshift pair of shift.rs:11-26 when centred = 1.  d_out may
 * equal d_in.  engine 0: SIMT mixed-radix FFT in FP32; engine 1: the DFT as
 * one GEMM on the tcgen05 tensor cores, split precision 3xBF16 with FP32
 * accumulation (n <= 2048; OKS_ENOTSUP beyond). */
int okscuda_dft_rows(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, long long nrows, int n,
                     int inverse, int centred, int engine);
/* Reads and clears the tensor-core kernels' error flag (synchronises the
 * context stream): 0 = no bounded wait ran out since the last read.  No
 * reference counterpart. */
int okscuda_tc_status(okscuda_ctx* ctx, int* status);
/* Bounds-checked build only (libokscuda_bounds.so, compiled with
 * -DOKS_BOUNDS_CHECK): ORs the error words of every kernel unit into *word
 * after synchronising the device (bit 1 exchange buffer, 2 staging buffer,
 * 4 column tile; 0 = no index ran out of range) and clears them when `clear`
 * is set.  The normal build returns OKS_ENOTSUP.  No reference counterpart. */
int okscuda_debug_bounds(okscuda_ctx* ctx, unsigned int* word, int clear);
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

/* strategy.rs:849-885 for a whole volume in one batched launch: placed
 * k-space d_kspace[nc, nz, ny, nx], per-slice host masks h_mask[nz, ny, nx],
 * per-coil FISTA, f32 RSS in coil order, centre crop to [ty, tx] per slice
 * (crop.rs:13-27 centring) into d_rss[nz, ty, tx].  d_coils[nc, nz, ny, nx]
 * receives the coil images when not NULL. */
int okscuda_cs_volume(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc,
                      int nz, int ny, int nx, int iters, float lambda, int ty, int tx, float* d_rss,
                      okscuda_c64* d_coils);

/* A list of independent slices of uneven size, coil count, iteration count,
 * lambda and mask (strategy.rs:850-880 for each), solved together: one
 * launch of the register-resident column engine per column length, units
 * ordered longest-first, length groups on concurrent streams.  Slices with
 * masks that vary along kx take the per-slice path. */
typedef struct {
    const okscuda_c64* d_kspace;   /* [nc, ny, nx] placed k-space             */
    const uint8_t* h_mask;         /* [ny, nx] host mask                      */
    int nc, ny, nx, iters;
    float lambda;
    float* d_rss;                  /* [ny, nx] RSS output                     */
    okscuda_c64* d_coils;          /* [nc, ny, nx] coil images, or NULL       */
} okscuda_slice_req;
int okscuda_cs_batch(okscuda_ctx* ctx, const okscuda_slice_req* reqs, int n);

/* ------------------------------------------------------------ SENSE mode */
/* Extension mode (no counterpart in the reference's per-coil cs, which
 * cs.rs:23-26 leaves SENSE-CS as a follow-up): one coil-combined image per
 * slice, min 1/2 sum_c ||M F S_c x - y_c||^2 + lambda ||W x||_1 by FISTA with
 * step 1/L (warm start A^H y, threshold lambda/L, LL band untouched,
 * cs.rs:99-137 momentum).  Maps S_c: Walsh's method (sensitivity.rs:37-142,
 * window walsh_window, walsh_iters power steps) on the low-resolution images
 * of the ACS block (longest run of sampled ky rows, grappa.rs:50-87;
 * strategy.rs:658-669), normalised to unit root-sum-of-squares.  L = ||A||^2
 * by an FP64 power iteration (power_iters steps).  ky-only masks, nc <= 32.
 * Outputs |x| to d_mag[ny, nx]; optionally the maps d_maps[nc, ny, nx], the
 * image d_x[ny, nx] and L.  Synchronous (L is read back). */
int okscuda_sense_cs(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc, int ny, int nx,
                     int iters, float lambda, int walsh_window, int walsh_iters, int power_iters, float* d_mag,
                     okscuda_c64* d_maps, okscuda_c64* d_x, double* h_lipschitz);

/* -------------------------------------------------------- output writers */
/* openkspace-cli/src/main.rs:1147-1153 percentile(): the element at index
 * round(pct / 100 * (n - 1)) (f32, half away from zero, clamped to n - 1) of
 * d_vals[n] in ascending order, found on the device by radix select (exact,
 * no sort); 0 for n = 0.  Synchronous: the value lands in *h_out. */
int okscuda_percentile(okscuda_ctx* ctx, const float* d_vals, long long n, float pct, float* h_out);
/* main.rs:1095-1110 write_png_linear (gamma = 0) and main.rs:1112-1140
 * write_png_windowed (gamma = 1) pixel mapping on the device:
 * d_out[i] = round(clamp((v - lo) / (hi - lo), 0, 1)^g * 255) with g = 1 or
 * 0.9 and hi raised to at least lo + FLT_EPSILON. */
int okscuda_window_u8(okscuda_ctx* ctx, const float* d_img, long long n, float lo, float hi, int gamma,
                      uint8_t* d_out);
/* main.rs:1033-1074 write_nifti_volume: NIfTI-1 single file (.nii) of the
 * host volume h_vol[nz, ny, nx] (float32, x fastest): dim = [3, nx, ny, nz],
 * 1 mm voxels, vox_offset 352, no extensions.  Host only (no context). */
int okscuda_write_nifti(const float* h_vol, int nz, int ny, int nx, const char* path);
/* The 8-bit grayscale PNG the reference writes with image::save_buffer
 * (main.rs:1108, 1137): h_gray[height, width], zlib stream of stored deflate
 * blocks.  Host only (no context). */
int okscuda_write_png(const uint8_t* h_gray, int width, int height, const char* path);

/* -------------------------------------------------- SENSE unfold (sense) */
/* sense.rs:64-192 sense_unfold_1d and sense.rs:194-252 sense_gfactor_1d on
 * the device: per reduced voxel (y0, x), y0 < ny / r, the r x r system
 * (C^H C + ridge I) rho = r C^H a with C[c][k] = maps[c][y0 + k ny/r][x] and
 * a[c] = aliased[c][y0][x], solved through the Cholesky factor and its
 * triangular inverse of prewhiten.rs:148-210, in f32 in the reference's
 * order (no fused multiply-adds).  d_out[ny, nx] (complex, may be NULL) gets
 * rho at rows y0 + k ny/r, d_gfactor[ny, nx] (may be NULL) the g-factor;
 * voxels whose factorisation fails stay zero.  OKS_EINVAL for r < 1
 * (SenseError::BadAcceleration), OKS_ESHAPE when r does not divide ny
 * (IndivisibleNy), OKS_ENOTSUP for r > 8. */
int okscuda_sense_unfold(okscuda_ctx* ctx, const okscuda_c64* d_aliased, const okscuda_c64* d_maps, int nc, int ny,
                         int nx, int r, float ridge, okscuda_c64* d_out, float* d_gfactor);

/* ------------------------------------------------------- request server */
/* No counterpart in the reference (which reconstructs one file at a time).
 * A request is one slice (strategy.rs:850-880).  Admission is by an HBM
 * budget and an in-flight limit: okscuda_server_submit returns OKS_EAGAIN
 * when the request does not fit now.
 * Mode 0 (default): each admitted request runs its own upload -> FISTA ->
 * RSS -> download chain on one stream of a pool, so requests that arrive
 * while others run overlap with them on the GPU.
 * Mode 1 (continuous batching): the upload of an admitted request starts at
 * submission on the server's upload stream; a dispatcher thread takes every
 * queued request whenever one of the server's batch slots is free and runs
 * them as one batched pass (okscuda_cs_batch: readout transforms, one
 * column-engine launch per column length over the (coil, column pair) units
 * of all of them, RSS, downloads) on that slot's streams; requests that
 * arrive while batches run join the next one, and the slots' batches overlap
 * on the GPU.  Mode 1 uses the server's context from its own thread: other
 * work belongs on another context while such a server exists.
 * Results are the same in both modes and the same as the request solved
 * alone.  Host buffers of a request must stay valid until it completes
 * (pinned memory keeps the copies asynchronous).  submit / poll / wait /
 * stats are thread-safe. */
typedef struct okscuda_server okscuda_server;
typedef struct {
    int max_inflight;              /* 0: 32 (queued + running)                 */
    size_t hbm_budget_bytes;       /* 0: half the free device memory           */
    int n_streams;                 /* 0: 12 streams (mode 0), 6 batch slots (mode 1) */
    int mode;                      /* 0: stream per request, 1: continuous batching */
} okscuda_server_cfg;
typedef struct {
    const okscuda_c64* h_kspace;   /* [nc, ny, nx] host k-space, or NULL ...   */
    const okscuda_c64* d_kspace;   /* ... device k-space (left unmodified)     */
    const uint8_t* h_mask;         /* [ny, nx]                                 */
    int nc, ny, nx, iters;
    float lambda;
    float* h_rss;                  /* [ny, nx] host output                     */
    long long coil_stride;         /* elements from one coil plane of the input to
                                      the next (0: ny * nx); e.g. nz * ny * nx for
                                      slice z of a [nc, nz, ny, nx] volume     */
} okscuda_request;
int okscuda_server_create(okscuda_ctx* ctx, const okscuda_server_cfg* cfg, okscuda_server** out);
void okscuda_server_destroy(okscuda_server* srv);
int okscuda_server_submit(okscuda_server* srv, const okscuda_request* req, uint64_t* id);
/* *done = 1 once the request finished; returns its status then and forgets it. */
int okscuda_server_poll(okscuda_server* srv, uint64_t id, int* done);
/* Bounded wait: OKS_ETIMEDOUT after timeout_ms (< 0: no limit). */
int okscuda_server_wait(okscuda_server* srv, uint64_t id, int timeout_ms);
int okscuda_server_stats(okscuda_server* srv, long long* inflight, long long* completed, size_t* reserved_bytes);

/* No counterpart in the reference.  okscuda_cs_slice for callers that cannot
 * allocate device memory -- applications whose allocator owns all device
 * memory (a framework memory pool, or a scanner pipeline that reserves its
 * budget at start-up and forbids allocation later).  It allocates nothing:
 * coil images, FFT tables, momentum weights and the row mask live in one
 * fixed 16 MiB device array inside the library (held by every GPU that loads
 * it until exit), so nc * ny * nx * 8 must fit 16 MiB - 256 KiB and ny, nx
 * <= 2048 (else OKS_ENOTSUP).  ky-only masks only.  The caller still passes
 * d_kspace[nc, ny, nx] and d_rss[ny, nx].  The first call on a device looks
 * up the array's device address: make it before any stream capture.  All
 * calls share the array, so calls that overlap on the GPU race: serialise
 * them (one stream). */
int okscuda_cs_slice_noalloc(okscuda_ctx* ctx, const okscuda_c64* d_kspace, const uint8_t* h_mask, int nc,
                             int ny, int nx, int iters, float lambda, float* d_rss);

/* ------------------------------------------------------- feeding stages */
/* prewhiten.rs:48-111 + 148-210 in FP64 on the device.  d_noise[nc, ns] holds
 * the samples of every noise scan with nc channels (concatenated along
 * samples); total_samples counts the samples of ALL noise scans, including
 * scans with another channel count, as prewhiten.rs:58 does (<= 0: use ns).
 * Writes W = L^-1 (complex64 [nc, nc], lower triangular) to d_W.  Synchronous.
 * OKS_ESKIP: total_samples < nc (prewhiten.rs:59-66); OKS_ENOTPD: Cholesky
 * pivot not finite or <= 0 (prewhiten.rs:161-164) -- the reference then
 * skips prewhitening. */
int okscuda_prewhiten_fit(okscuda_ctx* ctx, const okscuda_c64* d_noise, int nc, long long ns,
                          long long total_samples, okscuda_c64* d_W);
/* prewhiten.rs:118-142: every sample column of d_data[nacq, nc, ns] -> W s. */
int okscuda_prewhiten_apply(okscuda_ctx* ctx, const okscuda_c64* d_W, okscuda_c64* d_data, long long nacq,
                            int nc, int ns);
/* oversampling.rs:50-71 and 103-155: d_in[nlines, enc] -> d_out[nlines, rec]
 * (centred IFFT / enc, crop, centred FFT).  OKS_ESKIP when (enc, rec) is not
 * an integer ratio in 2..8 (the reference builds no remover). */
int okscuda_os_remove(okscuda_ctx* ctx, const okscuda_c64* d_in, okscuda_c64* d_out, long long nlines, int enc,
                      int rec);
/* fft.rs:52-56 ifft1_inplace(axis = 1): centred 1-D IFFT (1/nz) along kz of
 * d_data[nc, nz, ny, nx], in place (3-D decoupling, strategy.rs:824-827). */
int okscuda_ifft1_kz(okscuda_ctx* ctx, okscuda_c64* d_data, int nc, int nz, int ny, int nx);
/* fft.rs:19-29 ifft2_inplace on the last two axes of d_data[batch, ny, nx]
 * (1/ny and 1/nx), in place -- the odd-size fallback of strategy.rs:829-842. */
int okscuda_ifft2(okscuda_ctx* ctx, okscuda_c64* d_data, long long batch, int ny, int nx);

/* ------------------------------------------------ CsRss (strategy.rs:736-892) */
/* One acquisition (ISMRMRD AcquisitionHeader fields the cs path reads,
 * acquisition.rs:33-95).  Its samples are [active_channels, number_of_samples]
 * at data + data_offset. */
typedef struct {
    uint64_t flags;                 /* ISMRMRD flag bits (1 << (pos - 1))           */
    uint16_t number_of_samples;
    uint16_t active_channels;
    uint16_t discard_pre;
    uint16_t discard_post;
    uint16_t center_sample;
    uint16_t kspace_encode_step_1;
    uint16_t kspace_encode_step_2;
    uint16_t slice;
    uint16_t segment;               /* idx.segment: echo of a train (navigator bins) */
    long long data_offset;          /* in complex samples                          */
} okscuda_acq_header;

/* The reference's IsmrmrdFile as the cs path sees it. */
typedef struct {
    long long n_acq;
    const okscuda_acq_header* headers;   /* host [n_acq]                          */
    const okscuda_c64* data;             /* all samples (host, or device if flagged) */
    long long data_len;                  /* complex samples in data               */
    int data_on_device;                  /* 1: data is a device pointer           */
    int enc_x, enc_y, enc_z;             /* encoding.encoded_matrix               */
    int rec_x, rec_y, rec_z;             /* encoding.recon_matrix                 */
    int ky_center, kz_center;            /* encoding limits centre (reader.rs:343-347) */
} okscuda_acq_set;

/* CsRss public fields (strategy.rs:753-761). */
typedef struct {
    int remove_oversampling;
    int prewhiten;
    int phase_correct;
    int iters;
    float lambda;
    int fft_mode;                        /* 0 Auto, 1 TwoD, 2 ThreeD (strategy.rs:72-79) */
    int crop_to_recon_matrix;
} okscuda_csrss_cfg;

/* strategy.rs:763-775 defaults: iters 60, lambda 0.01, everything on. */
void okscuda_csrss_default(okscuda_csrss_cfg* cfg);
/* "cs" (strategy.rs:778-780) */
const char* okscuda_csrss_name(void);
/* sizeof(okscuda_acq_header) and sizeof(okscuda_acq_set), for bindings that
 * mirror the two structs (host only, no device needed). */
size_t okscuda_acq_header_size(void);
size_t okscuda_acq_set_size(void);
/* CsRss::reconstruct (strategy.rs:782-891): calibration, prewhitening,
 * oversampling removal, placement (reader.rs:225-468), kz decoupling,
 * odd-size fallback, per-slice per-coil FISTA, RSS, crop.  Writes the
 * magnitude volume [nz, ny, nx] (after crop) to h_out (host, capacity
 * out_cap floats) and its shape to out_dims[3]; h_out == NULL queries the
 * shape only.  When acqs->data_on_device is set, h_out is a device buffer
 * too and the call returns without waiting for the GPU.  OKS_EINVAL mirrors
 * IoError::MissingField (no image acquisitions / zero channels).  With
 * phase_correct set, phase-correction scans (ACQ_IS_PHASECORR_DATA) are
 * binned by (slice, segment) and every image line is multiplied by its bin's
 * unit phasor after prewhitening and before oversampling removal
 * (phasecorr.rs:61-169, strategy.rs:807-815). */
int okscuda_csrss_reconstruct(okscuda_ctx* ctx, const okscuda_csrss_cfg* cfg, const okscuda_acq_set* acqs,
                              float* h_out, long long out_cap, int* out_dims);

/* ------------------------------------------------ acquisition ingest */
/* IsmrmrdFile::open + the rows of /dataset/data (reader.rs:15-24, 47-76;
 * acquisition.rs:33-95; header.rs) without HDF5: the same rows serialised
 * as an acquisition stream file --
 *   "OKSACQ1\0", u32 xml_len, the ISMRMRD XML header, u64 n_acq, then per
 *   acquisition the packed 340-byte little-endian AcquisitionHeader (field
 *   order of acquisition.rs:33-59), f32 traj[trajectory_dimensions *
 *   number_of_samples], f32 data[2 * active_channels * number_of_samples].
 * okscuda_raw_open reads the headers, then the samples straight into one
 * pinned host buffer (ordinary memory when no device is present), and parses
 * the XML for the encoded / recon matrix sizes and the ky / kz encoding
 * centres (header.rs:128-206 tag-path rules).  OKS_EINVAL for an unreadable
 * or malformed file (IoError).  Host only (no context). */
typedef struct okscuda_raw okscuda_raw;
int okscuda_raw_open(const char* path, okscuda_raw** out);
/* The okscuda_acq_set of an open file (valid until okscuda_raw_close). */
int okscuda_raw_acq_set(const okscuda_raw* raw, okscuda_acq_set* out);
/* acquisitionSystemInformation/receiverChannels and the XML length. */
int okscuda_raw_info(const okscuda_raw* raw, int* receiver_channels, int* xml_len);
void okscuda_raw_close(okscuda_raw* raw);

/* ------------------------------------------------------------- profiling */
/* No reference counterpart (the reference has no timing hooks).  When
 * enabled, every kernel launch of this context is bracketed by CUDA events
 * on the context stream; okscuda_profile_read aggregates per kernel name the
 * summed device time (ms) and the launch count.  A replayed CUDA graph of the
 * 2-D engine is one entry, "k2d_graph", whose count is the kernel nodes it
 * ran.  Enabling clears the log. */
int okscuda_profile_enable(okscuda_ctx* ctx, int on);
int okscuda_profile_read(okscuda_ctx* ctx, char* names, int name_len, double* total_ms,
                         long long* launches, int nslots, int* nfound);

#ifdef __cplusplus
}
#endif
#endif /* OKSCUDA_H */
