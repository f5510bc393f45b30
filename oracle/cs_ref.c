/*
 * FP32 C restatement of OpenKSpace's `cs` path -- TEST INFRASTRUCTURE ONLY.
 *
 * Stand-in for the reference's own `cs` output (the reference is Rust and
 * cannot be built here) and the timed CPU baseline of the benchmark.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Each routine follows the reference routine it names (paths relative to
 * crates/openkspace-recon/src/): the same operation order, f32 throughout,
 * no FMA contraction (built with -ffp-contract=off, as rustc does not
 * contract).  The 1-D FFT is this file's own mixed-radix Stockham FFT; the
 * reference uses the un-vendored crate rustfft 6.4.1, whose exact rounding
 * is not reproduced (bit-level FFT parity is unpinned; the 1e-4 relative-L2
 * tolerance of the parity tests covers any accurate FFT).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float re, im; } cf;

static inline cf cadd(cf a, cf b) { cf r = {a.re + b.re, a.im + b.im}; return r; }
static inline cf csub(cf a, cf b) { cf r = {a.re - b.re, a.im - b.im}; return r; }
/* num_complex Mul: (ac - bd) + i(ad + bc) */
static inline cf cmul(cf a, cf b) { cf r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cf cscale(cf a, float s) { cf r = {a.re * s, a.im * s}; return r; }

/* ------------------------------------------------------------------------
 * Mixed-radix Stockham FFT (unnormalised), any n >= 1.
 * Stage with radix r, p = product of earlier radices: butterfly i in [0,n/r),
 * k = i mod p, inputs x[i + j n/r] * w_{pr}^{jk}, r-point DFT, outputs to
 * y[(i - k) r + k + j p].
 * ------------------------------------------------------------------------ */
typedef struct {
    int n, nst, sign;
    int rad[40], p[40];
    cf *tw[40];       /* per stage: tw[k*(r-1) + j-1] = w_{pr}^{jk}, j>=1 */
    cf *rtw[40];      /* per stage: r-th roots w_r^{m} for the generic radix */
    cf *buf;
} fftplan;

static void plan_free(fftplan *pl) {
    if (!pl) return;
    for (int s = 0; s < pl->nst; ++s) { free(pl->tw[s]); free(pl->rtw[s]); }
    free(pl->buf);
    free(pl);
}

static fftplan *plan_make(int n, int sign) {
    fftplan *pl = (fftplan *)calloc(1, sizeof(fftplan));
    pl->n = n; pl->sign = sign;
    int m = n, ns = 0;
    while (m % 4 == 0) { pl->rad[ns++] = 4; m /= 4; }
    while (m % 2 == 0) { pl->rad[ns++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { pl->rad[ns++] = f; m /= f; }
        if (f * f > m && m > 1) { pl->rad[ns++] = m; m = 1; }
    }
    pl->nst = ns;
    int p = 1;
    for (int s = 0; s < ns; ++s) {
        int r = pl->rad[s];
        pl->p[s] = p;
        pl->tw[s] = (cf *)malloc(sizeof(cf) * (size_t)(p * (r - 1) + 1));
        for (int k = 0; k < p; ++k)
            for (int j = 1; j < r; ++j) {
                double a = sign * 2.0 * M_PI * (double)j * (double)k / (double)(p * r);
                pl->tw[s][k * (r - 1) + j - 1].re = (float)cos(a);
                pl->tw[s][k * (r - 1) + j - 1].im = (float)sin(a);
            }
        pl->rtw[s] = (cf *)malloc(sizeof(cf) * (size_t)r);
        for (int q = 0; q < r; ++q) {
            double a = sign * 2.0 * M_PI * (double)q / (double)r;
            pl->rtw[s][q].re = (float)cos(a);
            pl->rtw[s][q].im = (float)sin(a);
        }
        p *= r;
    }
    pl->buf = (cf *)malloc(sizeof(cf) * (size_t)(n > 0 ? n : 1));
    return pl;
}

/* One transform of length n, in place on x (uses pl->buf as ping-pong). */
static void fft_exec(fftplan *pl, cf *x) {
    int n = pl->n;
    if (n <= 1) return;
    cf *src = x, *dst = pl->buf;
    const float sg = (float)pl->sign;
    const float s3 = 0.86602540378443864676f;
    const float c51 = 0.30901699437494742410f, c52 = -0.80901699437494742410f;
    const float s51 = 0.95105651629515357212f, s52 = 0.58778525229247312917f;
    for (int s = 0; s < pl->nst; ++s) {
        int r = pl->rad[s], p = pl->p[s], nb = n / r;
        const cf *tw = pl->tw[s];
        for (int i = 0; i < nb; ++i) {
            int k = i % p;
            cf v[64];
            int base = (i - k) * r + k;
            if (r <= 64) {
                v[0] = src[i];
                for (int j = 1; j < r; ++j) v[j] = cmul(src[i + j * nb], tw[k * (r - 1) + j - 1]);
            }
            if (r == 2) {
                dst[base] = cadd(v[0], v[1]);
                dst[base + p] = csub(v[0], v[1]);
            } else if (r == 4) {
                cf a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
                cf c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
                /* forward: w4 = -i ; d * (sign i) */
                cf di = {-sg * d.im, sg * d.re};
                dst[base] = cadd(a, c);
                dst[base + p] = cadd(b, di);
                dst[base + 2 * p] = csub(a, c);
                dst[base + 3 * p] = csub(b, di);
            } else if (r == 3) {
                cf t1 = cadd(v[1], v[2]);
                cf t2 = {v[0].re - 0.5f * t1.re, v[0].im - 0.5f * t1.im};
                cf d = csub(v[1], v[2]);
                cf t3 = {-sg * s3 * d.im, sg * s3 * d.re};
                dst[base] = cadd(v[0], t1);
                dst[base + p] = cadd(t2, t3);
                dst[base + 2 * p] = csub(t2, t3);
            } else if (r == 5) {
                cf a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
                cf a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
                cf t1 = {v[0].re + c51 * a1.re + c52 * a2.re, v[0].im + c51 * a1.im + c52 * a2.im};
                cf t2 = {v[0].re + c52 * a1.re + c51 * a2.re, v[0].im + c52 * a1.im + c51 * a2.im};
                cf u1 = {s51 * b1.re + s52 * b2.re, s51 * b1.im + s52 * b2.im};
                cf u2 = {s52 * b1.re - s51 * b2.re, s52 * b1.im - s51 * b2.im};
                cf iu1 = {-sg * u1.im, sg * u1.re}, iu2 = {-sg * u2.im, sg * u2.re};
                dst[base] = cadd(cadd(v[0], a1), a2);
                dst[base + p] = cadd(t1, iu1);
                dst[base + 4 * p] = csub(t1, iu1);
                dst[base + 2 * p] = cadd(t2, iu2);
                dst[base + 3 * p] = csub(t2, iu2);
            } else {
                /* generic radix: direct DFT, O(r^2) */
                const cf *w = pl->rtw[s];
                for (int q = 0; q < r; ++q) {
                    cf acc = {0.f, 0.f};
                    for (int j = 0; j < r; ++j) {
                        cf vj = (r <= 64) ? v[j]
                                          : (j == 0 ? src[i] : cmul(src[i + j * nb], tw[k * (r - 1) + j - 1]));
                        acc = cadd(acc, cmul(vj, w[(int)(((long)q * j) % r)]));
                    }
                    dst[base + q * p] = acc;
                }
            }
        }
        cf *t = src; src = dst; dst = t;
    }
    if (src != x) memcpy(x, src, sizeof(cf) * (size_t)n);
}

/* ------------------------------------------------------------------------
 * shift.rs: rotate a strided lane left by k (np.roll by -k)
 * ------------------------------------------------------------------------ */
static void rotate_lane(cf *a, int n, long stride, int k, cf *tmp) {
    if (n < 2 || k == 0 || k >= n) return;
    for (int i = 0; i < n; ++i) tmp[i] = a[(long)i * stride];
    for (int i = 0; i < n; ++i) a[(long)i * stride] = tmp[(i + k) % n];
}

/* rotate every lane of [ny, nx] along axis (0 = y, 1 = x) */
static void rotate2(cf *a, int ny, int nx, int axis, int k, cf *tmp) {
    if (axis == 0)
        for (int x = 0; x < nx; ++x) rotate_lane(a + x, ny, nx, k, tmp);
    else
        for (int y = 0; y < ny; ++y) rotate_lane(a + (long)y * nx, nx, 1, k, tmp);
}

typedef struct {
    int ny, nx;
    fftplan *fx, *fy, *ix, *iy;
    cf *row, *col, *tmp;
} cs_work;

static cs_work *work_make(int ny, int nx) {
    cs_work *w = (cs_work *)calloc(1, sizeof(cs_work));
    w->ny = ny; w->nx = nx;
    w->fx = plan_make(nx, -1); w->fy = plan_make(ny, -1);
    w->ix = plan_make(nx, +1); w->iy = plan_make(ny, +1);
    int m = ny > nx ? ny : nx;
    w->row = (cf *)malloc(sizeof(cf) * (size_t)m);
    w->col = (cf *)malloc(sizeof(cf) * (size_t)m);
    w->tmp = (cf *)malloc(sizeof(cf) * (size_t)m);
    return w;
}

static void work_free(cs_work *w) {
    plan_free(w->fx); plan_free(w->fy); plan_free(w->ix); plan_free(w->iy);
    free(w->row); free(w->col); free(w->tmp); free(w);
}

/* cs.rs:141-218 centred_fft2 / centred_ifft2 */
static void centred_2d(cs_work *w, cf *a, int inverse) {
    int ny = w->ny, nx = w->nx;
    fftplan *px = inverse ? w->ix : w->fx, *py = inverse ? w->iy : w->fy;
    rotate2(a, ny, nx, 0, (ny + 1) / 2, w->tmp);
    rotate2(a, ny, nx, 1, (nx + 1) / 2, w->tmp);
    for (int i = 0; i < ny; ++i) {
        memcpy(w->row, a + (long)i * nx, sizeof(cf) * (size_t)nx);
        fft_exec(px, w->row);
        memcpy(a + (long)i * nx, w->row, sizeof(cf) * (size_t)nx);
    }
    for (int j = 0; j < nx; ++j) {
        for (int i = 0; i < ny; ++i) w->col[i] = a[(long)i * nx + j];
        fft_exec(py, w->col);
        for (int i = 0; i < ny; ++i) a[(long)i * nx + j] = w->col[i];
    }
    rotate2(a, ny, nx, 0, ny / 2, w->tmp);
    rotate2(a, ny, nx, 1, nx / 2, w->tmp);
    float s = 1.0f / sqrtf((float)ny * (float)nx);
    for (long q = 0; q < (long)ny * nx; ++q) a[q] = cscale(a[q], s);
}

/* wavelet.rs:32-52 */
static void haar_fwd(const cf *x, cf *out, int ny, int nx) {
    int hy = ny / 2, hx = nx / 2;
    for (int i = 0; i < hy; ++i)
        for (int j = 0; j < hx; ++j) {
            cf a = x[(long)(2 * i) * nx + 2 * j], b = x[(long)(2 * i) * nx + 2 * j + 1];
            cf d = x[(long)(2 * i + 1) * nx + 2 * j], e = x[(long)(2 * i + 1) * nx + 2 * j + 1];
            out[(long)i * nx + j] = cscale(cadd(cadd(cadd(a, b), d), e), 0.5f);
            out[(long)i * nx + hx + j] = cscale(csub(cadd(csub(a, b), d), e), 0.5f);
            out[(long)(hy + i) * nx + j] = cscale(csub(csub(cadd(a, b), d), e), 0.5f);
            out[(long)(hy + i) * nx + hx + j] = cscale(cadd(csub(csub(a, b), d), e), 0.5f);
        }
}

/* wavelet.rs:55-75 */
static void haar_inv(const cf *y, cf *out, int ny, int nx) {
    int hy = ny / 2, hx = nx / 2;
    for (int i = 0; i < hy; ++i)
        for (int j = 0; j < hx; ++j) {
            cf ll = y[(long)i * nx + j], hl = y[(long)i * nx + hx + j];
            cf lh = y[(long)(hy + i) * nx + j], hh = y[(long)(hy + i) * nx + hx + j];
            out[(long)(2 * i) * nx + 2 * j] = cscale(cadd(cadd(cadd(ll, hl), lh), hh), 0.5f);
            out[(long)(2 * i) * nx + 2 * j + 1] = cscale(csub(cadd(csub(ll, hl), lh), hh), 0.5f);
            out[(long)(2 * i + 1) * nx + 2 * j] = cscale(csub(csub(cadd(ll, hl), lh), hh), 0.5f);
            out[(long)(2 * i + 1) * nx + 2 * j + 1] = cscale(cadd(csub(csub(ll, hl), lh), hh), 0.5f);
        }
}

/* wavelet.rs:80-99 (norm() = hypot) */
static void shrink_details(cf *y, int ny, int nx, float lambda) {
    int hy = ny / 2, hx = nx / 2;
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            if (i < hy && j < hx) continue;
            cf z = y[(long)i * nx + j];
            float m = hypotf(z.re, z.im);
            if (m <= lambda) {
                y[(long)i * nx + j].re = 0.f;
                y[(long)i * nx + j].im = 0.f;
            } else {
                float s = (m - lambda) / m;
                y[(long)i * nx + j] = cscale(z, s);
            }
        }
}

/* cs.rs:59-139 with work buffers provided */
static int fista_w(cs_work *w, const cf *k, const uint8_t *mask, int iters, float lambda, cf *out) {
    int ny = w->ny, nx = w->nx;
    long N = (long)ny * nx;
    if (ny % 2 || nx % 2) return -3;
    cf *atb = (cf *)malloc(sizeof(cf) * N), *x = (cf *)malloc(sizeof(cf) * N);
    cf *z = (cf *)malloc(sizeof(cf) * N), *az = (cf *)malloc(sizeof(cf) * N);
    cf *coef = (cf *)malloc(sizeof(cf) * N), *xn = (cf *)malloc(sizeof(cf) * N);
    for (long q = 0; q < N; ++q) {
        atb[q] = k[q];
        if (!mask[q]) { atb[q].re = 0.f; atb[q].im = 0.f; }
    }
    centred_2d(w, atb, 1);
    memcpy(x, atb, sizeof(cf) * N);
    memcpy(z, x, sizeof(cf) * N);
    float t = 1.0f;
    for (int it = 0; it < iters; ++it) {
        memcpy(az, z, sizeof(cf) * N);
        centred_2d(w, az, 0);
        for (long q = 0; q < N; ++q) {
            if (mask[q]) az[q] = csub(az[q], k[q]);
            else { az[q].re = 0.f; az[q].im = 0.f; }
        }
        centred_2d(w, az, 1);
        for (long q = 0; q < N; ++q) az[q] = csub(z[q], az[q]);   /* v */
        haar_fwd(az, coef, ny, nx);
        shrink_details(coef, ny, nx, lambda);
        haar_inv(coef, xn, ny, nx);
        float t_new = 0.5f * (1.0f + sqrtf(1.0f + 4.0f * t * t));
        float alpha = (t - 1.0f) / t_new;
        cf ca = {alpha, 0.f};
        for (long q = 0; q < N; ++q) z[q] = cadd(xn[q], cmul(ca, csub(xn[q], x[q])));
        memcpy(x, xn, sizeof(cf) * N);
        t = t_new;
    }
    memcpy(out, x, sizeof(cf) * N);
    free(atb); free(x); free(z); free(az); free(coef); free(xn);
    return 0;
}

/* ------------------------------------------------------------------------
 * exported API (interleaved re/im float pairs)
 * ------------------------------------------------------------------------ */
int csref_fft_1d(float *data, int n, int howmany, int inverse) {
    fftplan *pl = plan_make(n, inverse ? +1 : -1);
    for (int h = 0; h < howmany; ++h) fft_exec(pl, (cf *)data + (long)h * n);
    plan_free(pl);
    return 0;
}

int csref_centred_fft2(float *a, int ny, int nx, int howmany, int inverse) {
    cs_work *w = work_make(ny, nx);
    for (int h = 0; h < howmany; ++h) centred_2d(w, (cf *)a + (long)h * ny * nx, inverse);
    work_free(w);
    return 0;
}

int csref_haar_forward(const float *in, float *out, int ny, int nx) {
    if (ny % 2 || nx % 2) return -3;
    haar_fwd((const cf *)in, (cf *)out, ny, nx);
    return 0;
}

int csref_haar_inverse(const float *in, float *out, int ny, int nx) {
    if (ny % 2 || nx % 2) return -3;
    haar_inv((const cf *)in, (cf *)out, ny, nx);
    return 0;
}

int csref_soft_threshold_details(float *y, int ny, int nx, float lambda) {
    shrink_details((cf *)y, ny, nx, lambda);
    return 0;
}

int csref_fista_cs_single_coil(const float *k, const uint8_t *mask, int ny, int nx,
                               int iters, float lambda, float *out) {
    if (ny % 2 || nx % 2) return -3;
    cs_work *w = work_make(ny, nx);
    int rc = fista_w(w, (const cf *)k, mask, iters, lambda, (cf *)out);
    work_free(w);
    return rc;
}

/* strategy.rs:849-880: per slice, per coil FISTA, then f32 RSS in coil order.
 * Work items (slice, coil) are spread over nthreads threads. */
typedef struct {
    const cf *k; const uint8_t *mask; int nc, nz, ny, nx, iters; float lambda;
    cf *coils; volatile int next; pthread_mutex_t mu; int rc;
} csrss_job;

static void *csrss_worker(void *arg) {
    csrss_job *J = (csrss_job *)arg;
    cs_work *w = work_make(J->ny, J->nx);
    long N = (long)J->ny * J->nx;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        int item = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (item >= J->nc * J->nz) break;
        int kz = item / J->nc, c = item % J->nc;
        const cf *kin = J->k + ((long)c * J->nz + kz) * N;
        int rc = fista_w(w, kin, J->mask + (long)kz * N, J->iters, J->lambda,
                         J->coils + ((long)c * J->nz + kz) * N);
        if (rc) J->rc = rc;
    }
    work_free(w);
    return NULL;
}

int csref_csrss(const float *kspace, const uint8_t *mask, int nc, int nz, int ny, int nx,
                int iters, float lambda, int nthreads, float *out_rss, float *out_coils) {
    if (ny % 2 || nx % 2) return -3;
    long N = (long)ny * nx;
    cf *coils = out_coils ? (cf *)out_coils : (cf *)malloc(sizeof(cf) * (size_t)nc * nz * N);
    csrss_job J;
    memset(&J, 0, sizeof(J));
    J.k = (const cf *)kspace; J.mask = mask; J.nc = nc; J.nz = nz; J.ny = ny; J.nx = nx;
    J.iters = iters; J.lambda = lambda; J.coils = coils; J.next = 0;
    pthread_mutex_init(&J.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    pthread_t th[256];
    if (nthreads > 256) nthreads = 256;
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, csrss_worker, &J);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&J.mu);
    for (int kz = 0; kz < nz; ++kz)
        for (long q = 0; q < N; ++q) {
            float s = 0.f;
            for (int c = 0; c < nc; ++c) {
                cf v = coils[((long)c * nz + kz) * N + q];
                s += v.re * v.re + v.im * v.im;   /* norm_sqr */
            }
            out_rss[(long)kz * N + q] = sqrtf(s);
        }
    if (!out_coils) free(coils);
    return J.rc;
}

/* prewhiten.rs:48-111, 148-210 (f32).  noise is one [nc, ns] block.
 * Returns 0 and W (lower triangular, [nc, nc]) or 1 when skipped (too few
 * samples / not positive definite / singular). */
int csref_prewhiten_fit(const float *noise, int nc, long ns, float *W) {
    if (nc <= 0 || ns < nc) return 1;
    const cf *s = (const cf *)noise;
    cf *psi = (cf *)calloc((size_t)nc * nc, sizeof(cf));
    for (long n = 0; n < ns; ++n)
        for (int i = 0; i < nc; ++i) {
            cf si = s[(long)i * ns + n];
            for (int j = 0; j < nc; ++j) {
                cf sj = s[(long)j * ns + n];
                cf cj = {sj.re, -sj.im};
                psi[i * nc + j] = cadd(psi[i * nc + j], cmul(si, cj));
            }
        }
    float denom = (float)ns - 1.0f;
    if (denom < 1.0f) denom = 1.0f;
    for (int q = 0; q < nc * nc; ++q) { psi[q].re /= denom; psi[q].im /= denom; }
    cf *l = (cf *)calloc((size_t)nc * nc, sizeof(cf));
    int rc = 0;
    for (int i = 0; i < nc && !rc; ++i) {
        cf diag = psi[i * nc + i];
        for (int k = 0; k < i; ++k) {
            cf lk = l[i * nc + k], ck = {lk.re, -lk.im};
            diag = csub(diag, cmul(lk, ck));
        }
        float d_re = diag.re;
        if (!isfinite(d_re) || d_re <= 0.0f) { rc = 1; break; }
        float lii = sqrtf(d_re);
        l[i * nc + i].re = lii; l[i * nc + i].im = 0.f;
        float inv = 1.0f / lii;
        for (int j = i + 1; j < nc; ++j) {
            cf sj = psi[j * nc + i];
            for (int k = 0; k < i; ++k) {
                cf lik = l[i * nc + k], c = {lik.re, -lik.im};
                sj = csub(sj, cmul(l[j * nc + k], c));
            }
            cf iv = {inv, 0.f};
            l[j * nc + i] = cmul(sj, iv);
        }
    }
    cf *o = (cf *)W;
    if (!rc) {
        memset(o, 0, sizeof(cf) * (size_t)nc * nc);
        for (int col = 0; col < nc && !rc; ++col)
            for (int i = 0; i < nc; ++i) {
                cf sacc = {i == col ? 1.f : 0.f, 0.f};
                for (int j = 0; j < i; ++j) sacc = csub(sacc, cmul(l[i * nc + j], o[j * nc + col]));
                cf d = l[i * nc + i];
                if (fabsf(d.re) < 1.1920929e-7f && fabsf(d.im) < 1.1920929e-7f) { rc = 1; break; }
                /* num_complex Div */
                float den = d.re * d.re + d.im * d.im;
                cf q = {(sacc.re * d.re + sacc.im * d.im) / den, (sacc.im * d.re - sacc.re * d.im) / den};
                o[i * nc + col] = q;
            }
        for (int i = 0; i < nc; ++i)
            for (int j = i + 1; j < nc; ++j) { o[i * nc + j].re = 0.f; o[i * nc + j].im = 0.f; }
    }
    free(psi); free(l);
    return rc;
}

/* prewhiten.rs:118-142: data [nacq][nc][ns], each sample column s -> W s */
int csref_prewhiten_apply(const float *W, float *data, long nacq, int nc, int ns) {
    const cf *w = (const cf *)W;
    cf *buf = (cf *)malloc(sizeof(cf) * (size_t)nc);
    for (long a = 0; a < nacq; ++a) {
        cf *d = (cf *)data + a * (long)nc * ns;
        for (int n = 0; n < ns; ++n) {
            for (int i = 0; i < nc; ++i) buf[i] = d[(long)i * ns + n];
            for (int i = 0; i < nc; ++i) {
                cf acc = {0.f, 0.f};
                for (int j = 0; j <= i; ++j) acc = cadd(acc, cmul(w[i * nc + j], buf[j]));
                d[(long)i * ns + n] = acc;
            }
        }
    }
    free(buf);
    return 0;
}

/* oversampling.rs:103-155: in [nacq][nc][enc] -> out [nacq][nc][rec] */
int csref_os_apply(const float *in, float *out, long nacq, int nc, int enc, int rec) {
    if (rec == 0 || enc <= rec || enc % rec != 0 || enc / rec > 8) return -1;
    fftplan *pi = plan_make(enc, +1), *pf = plan_make(rec, -1);
    cf *lane = (cf *)malloc(sizeof(cf) * (size_t)enc), *tmp = (cf *)malloc(sizeof(cf) * (size_t)enc);
    cf *crop = (cf *)malloc(sizeof(cf) * (size_t)rec);
    float sc = 1.0f / (float)enc;
    int start = (enc - rec) / 2;
    for (long a = 0; a < nacq * nc; ++a) {
        memcpy(lane, (const cf *)in + a * enc, sizeof(cf) * (size_t)enc);
        rotate_lane(lane, enc, 1, (enc + 1) / 2, tmp);
        fft_exec(pi, lane);
        for (int i = 0; i < enc; ++i) lane[i] = cscale(lane[i], sc);
        rotate_lane(lane, enc, 1, enc / 2, tmp);
        memcpy(crop, lane + start, sizeof(cf) * (size_t)rec);
        rotate_lane(crop, rec, 1, (rec + 1) / 2, tmp);
        fft_exec(pf, crop);
        rotate_lane(crop, rec, 1, rec / 2, tmp);
        memcpy((cf *)out + a * rec, crop, sizeof(cf) * (size_t)rec);
    }
    free(lane); free(tmp); free(crop);
    plan_free(pi); plan_free(pf);
    return 0;
}

/* fft.rs:52-84: centred 1-D IFFT (1/n) along the middle axis of
 * [n_outer][n][n_inner] */
int csref_ifft1_axis(float *data, long n_outer, int n, long n_inner) {
    if (n < 2) return 0;
    fftplan *pl = plan_make(n, +1);
    cf *lane = (cf *)malloc(sizeof(cf) * (size_t)n), *tmp = (cf *)malloc(sizeof(cf) * (size_t)n);
    float norm = 1.0f / (float)n;
    for (long o = 0; o < n_outer; ++o)
        for (long q = 0; q < n_inner; ++q) {
            cf *a = (cf *)data + o * (long)n * n_inner + q;
            rotate_lane(a, n, n_inner, (n + 1) / 2, tmp);
            for (int i = 0; i < n; ++i) lane[i] = a[(long)i * n_inner];
            fft_exec(pl, lane);
            for (int i = 0; i < n; ++i) a[(long)i * n_inner] = cscale(lane[i], norm);
            rotate_lane(a, n, n_inner, n / 2, tmp);
        }
    free(lane); free(tmp);
    plan_free(pl);
    return 0;
}

/* sense.rs:64-252 sense_unfold_1d / sense_gfactor_1d (f32, the reference's
 * order; Cholesky and inverse as prewhiten.rs:148-210).  aliased, maps:
 * [nc, ny, nx]; out [ny, nx] (may be NULL), g [ny, nx] (may be NULL); voxels
 * whose factorisation fails stay zero.  Returns 1 for R < 1 or ny % R != 0. */
int csref_sense_unfold(const float *aliased, const float *maps, int nc, int ny, int nx, int r, float ridge,
                       float *out, float *g) {
    if (r < 1 || ny % r) return 1;
    const cf *al = (const cf *)aliased, *mp = (const cf *)maps;
    cf *o = (cf *)out;
    const long plane = (long)ny * nx;
    if (o) memset(o, 0, sizeof(cf) * (size_t)plane);
    if (g) memset(g, 0, sizeof(float) * (size_t)plane);
    const int nyr = ny / r;
    if (nc == 0 || nx == 0 || nyr == 0) return 0;
    cf *C = (cf *)malloc(sizeof(cf) * (size_t)nc * r);
    cf *chc = (cf *)malloc(sizeof(cf) * (size_t)r * r);
    cf *l = (cf *)malloc(sizeof(cf) * (size_t)r * r);
    cf *inv = (cf *)malloc(sizeof(cf) * (size_t)r * r);
    cf *rhs = (cf *)malloc(sizeof(cf) * (size_t)r);
    cf *tmp = (cf *)malloc(sizeof(cf) * (size_t)r);
    for (int x = 0; x < nx; ++x)
        for (int y0 = 0; y0 < nyr; ++y0) {
            for (int c = 0; c < nc; ++c)
                for (int k = 0; k < r; ++k) C[c * r + k] = mp[c * plane + (long)(y0 + k * nyr) * nx + x];
            for (int a = 0; a < r; ++a)
                for (int b = 0; b < r; ++b) {
                    cf acc = {0.f, 0.f};
                    for (int c = 0; c < nc; ++c) {
                        cf ca = C[c * r + a], cc = {ca.re, -ca.im};
                        acc = cadd(acc, cmul(cc, C[c * r + b]));
                    }
                    if (a == b) { cf rd = {ridge, 0.f}; acc = cadd(acc, rd); }
                    chc[a * r + b] = acc;
                }
            for (int a = 0; a < r; ++a) {
                cf acc = {0.f, 0.f};
                for (int c = 0; c < nc; ++c) {
                    cf ca = C[c * r + a], cc = {ca.re, -ca.im};
                    acc = cadd(acc, cmul(cc, al[c * plane + (long)y0 * nx + x]));
                }
                cf rr = {(float)r, 0.f};
                rhs[a] = cmul(acc, rr);
            }
            int bad = 0;
            memset(l, 0, sizeof(cf) * (size_t)r * r);
            for (int i = 0; i < r && !bad; ++i) {
                cf diag = chc[i * r + i];
                for (int k = 0; k < i; ++k) {
                    cf lk = l[i * r + k], ck = {lk.re, -lk.im};
                    diag = csub(diag, cmul(lk, ck));
                }
                float d_re = diag.re;
                if (!isfinite(d_re) || d_re <= 0.0f) { bad = 1; break; }
                float lii = sqrtf(d_re);
                l[i * r + i].re = lii; l[i * r + i].im = 0.f;
                cf iv = {1.0f / lii, 0.f};
                for (int j = i + 1; j < r; ++j) {
                    cf s = chc[j * r + i];
                    for (int k = 0; k < i; ++k) {
                        cf lik = l[i * r + k], c2 = {lik.re, -lik.im};
                        s = csub(s, cmul(l[j * r + k], c2));
                    }
                    l[j * r + i] = cmul(s, iv);
                }
            }
            if (bad) continue;
            memset(inv, 0, sizeof(cf) * (size_t)r * r);
            for (int col = 0; col < r && !bad; ++col)
                for (int i = 0; i < r; ++i) {
                    cf s = {i == col ? 1.f : 0.f, 0.f};
                    for (int j = 0; j < i; ++j) s = csub(s, cmul(l[i * r + j], inv[j * r + col]));
                    cf d = l[i * r + i];
                    if (fabsf(d.re) < 1.1920929e-7f && fabsf(d.im) < 1.1920929e-7f) { bad = 1; break; }
                    float den = d.re * d.re + d.im * d.im;
                    cf q = {(s.re * d.re + s.im * d.im) / den, (s.im * d.re - s.re * d.im) / den};
                    inv[i * r + col] = q;
                }
            if (bad) continue;
            for (int i = 0; i < r; ++i)
                for (int j = i + 1; j < r; ++j) { inv[i * r + j].re = 0.f; inv[i * r + j].im = 0.f; }
            if (o) {
                for (int i = 0; i < r; ++i) {
                    cf acc = {0.f, 0.f};
                    for (int j = 0; j <= i; ++j) acc = cadd(acc, cmul(inv[i * r + j], rhs[j]));
                    tmp[i] = acc;
                }
                for (int i = 0; i < r; ++i) {
                    cf acc = {0.f, 0.f};
                    for (int j = i; j < r; ++j) {
                        cf v = inv[j * r + i], vc = {v.re, -v.im};
                        acc = cadd(acc, cmul(vc, tmp[j]));
                    }
                    o[(long)(y0 + i * nyr) * nx + x] = acc;
                }
            }
            if (g)
                for (int k = 0; k < r; ++k) {
                    float inv_diag = 0.f;
                    for (int j = k; j < r; ++j) {
                        cf v = inv[j * r + k];
                        inv_diag += v.re * v.re + v.im * v.im;
                    }
                    float cd = chc[k * r + k].re;
                    if (!(cd > 0.f)) cd = (cd != cd) ? 0.f : (cd > 0.f ? cd : 0.f);
                    float p = inv_diag * cd;
                    g[(long)(y0 + k * nyr) * nx + x] = sqrtf(p > 0.f ? p : 0.f);
                }
        }
    free(C); free(chc); free(l); free(inv); free(rhs); free(tmp);
    return 0;
}
