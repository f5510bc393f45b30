"""FP64 oracle: numpy complex128 restatement of OpenKSpace's ``cs`` path.

Test infrastructure only (see ``oracle/__init__.py``).  Every function follows
the reference routine it names, file:line relative to the reference project
(``crates/openkspace-recon/src/...``), with complex64 replaced by complex128.
Batch axes are allowed in front of the 2-D axes so a whole slice (all coils)
runs as one numpy call; the arithmetic per (slice, coil) is the reference's.
"""
from __future__ import annotations

import numpy as np

HAAR_NORM = 0.5  # wavelet.rs:27


# --------------------------------------------------------------------------
# shift.rs
# --------------------------------------------------------------------------
def _rotate_left(a: np.ndarray, axis: int, k: int) -> np.ndarray:
    """shift.rs:29-51 rotate_axis: lane[i] = buf[(i + k) % n] (np.roll by -k)."""
    n = a.shape[axis]
    if k == 0 or k >= n:
        return a.copy()
    return np.roll(a, -k, axis=axis)


def fftshift_axis(a: np.ndarray, axis: int) -> np.ndarray:
    """shift.rs:11-17: rotate left by n/2 (floor)."""
    n = a.shape[axis]
    if n < 2:
        return a.copy()
    return _rotate_left(a, axis, n // 2)


def ifftshift_axis(a: np.ndarray, axis: int) -> np.ndarray:
    """shift.rs:20-26: rotate left by ceil(n/2)."""
    n = a.shape[axis]
    if n < 2:
        return a.copy()
    return _rotate_left(a, axis, (n + 1) // 2)


# --------------------------------------------------------------------------
# cs.rs centred unitary 2-D FFT pair
# --------------------------------------------------------------------------
def centred_fft2(a: np.ndarray) -> np.ndarray:
    """cs.rs:141-178: ifftshift(y,x) -> DFT rows (x) -> DFT cols (y) ->
    fftshift(y,x) -> * 1/sqrt(ny*nx).  Operates on the last two axes."""
    ny, nx = a.shape[-2:]
    a = ifftshift_axis(np.asarray(a, dtype=np.complex128), -2)
    a = ifftshift_axis(a, -1)
    a = np.fft.fft(a, axis=-1)
    a = np.fft.fft(a, axis=-2)
    a = fftshift_axis(a, -2)
    a = fftshift_axis(a, -1)
    return a * (1.0 / np.sqrt(float(ny) * float(nx)))


def centred_ifft2(a: np.ndarray) -> np.ndarray:
    """cs.rs:180-218: as centred_fft2 with the unnormalised inverse DFT
    (e^{+}) and the same 1/sqrt(ny*nx) scale."""
    ny, nx = a.shape[-2:]
    a = ifftshift_axis(np.asarray(a, dtype=np.complex128), -2)
    a = ifftshift_axis(a, -1)
    a = np.fft.ifft(a, axis=-1) * nx  # rustfft inverse is unnormalised
    a = np.fft.ifft(a, axis=-2) * ny
    a = fftshift_axis(a, -2)
    a = fftshift_axis(a, -1)
    return a * (1.0 / np.sqrt(float(ny) * float(nx)))


# --------------------------------------------------------------------------
# wavelet.rs
# --------------------------------------------------------------------------
def haar_forward(x: np.ndarray) -> np.ndarray:
    """wavelet.rs:32-52: one-level Haar, quadrant layout LL|HL / LH|HH."""
    ny, nx = x.shape[-2:]
    if ny % 2 or nx % 2:
        raise ValueError("Haar: dims must be even")
    hy, hx = ny // 2, nx // 2
    a = x[..., 0::2, 0::2]
    b = x[..., 0::2, 1::2]
    d = x[..., 1::2, 0::2]
    e = x[..., 1::2, 1::2]
    out = np.empty(x.shape, dtype=np.result_type(x.dtype, np.complex128))
    out[..., :hy, :hx] = (a + b + d + e) * HAAR_NORM  # LL
    out[..., :hy, hx:] = (a - b + d - e) * HAAR_NORM  # HL
    out[..., hy:, :hx] = (a + b - d - e) * HAAR_NORM  # LH
    out[..., hy:, hx:] = (a - b - d + e) * HAAR_NORM  # HH
    return out


def haar_inverse(y: np.ndarray) -> np.ndarray:
    """wavelet.rs:55-75: exact inverse (= adjoint) of haar_forward."""
    ny, nx = y.shape[-2:]
    if ny % 2 or nx % 2:
        raise ValueError("Haar: dims must be even")
    hy, hx = ny // 2, nx // 2
    ll = y[..., :hy, :hx]
    hl = y[..., :hy, hx:]
    lh = y[..., hy:, :hx]
    hh = y[..., hy:, hx:]
    out = np.empty(y.shape, dtype=np.result_type(y.dtype, np.complex128))
    out[..., 0::2, 0::2] = (ll + hl + lh + hh) * HAAR_NORM
    out[..., 0::2, 1::2] = (ll - hl + lh - hh) * HAAR_NORM
    out[..., 1::2, 0::2] = (ll + hl - lh - hh) * HAAR_NORM
    out[..., 1::2, 1::2] = (ll - hl - lh + hh) * HAAR_NORM
    return out


def soft_threshold_details(y: np.ndarray, lam: float) -> np.ndarray:
    """wavelet.rs:80-99: complex soft-threshold of every coefficient outside
    the LL quadrant; |z| <= lambda -> 0, else z * (|z| - lambda) / |z|."""
    ny, nx = y.shape[-2:]
    hy, hx = ny // 2, nx // 2
    out = np.array(y, dtype=np.complex128, copy=True)
    m = np.abs(out)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.where(m <= lam, 0.0, (m - lam) / np.where(m == 0, 1.0, m))
    ll = out[..., :hy, :hx].copy()
    out *= s
    out[..., :hy, :hx] = ll
    return out


# --------------------------------------------------------------------------
# cs.rs FISTA
# --------------------------------------------------------------------------
def fista_alpha_table(iters: int, dtype=np.float64) -> np.ndarray:
    """cs.rs:125-126: t' = 0.5 (1 + sqrt(1 + 4 t^2)), alpha = (t - 1) / t',
    t0 = 1.  ``dtype=np.float32`` reproduces the reference's f32 recursion."""
    t = dtype(1.0)
    out = np.empty(iters, dtype=dtype)
    half, one, four = dtype(0.5), dtype(1.0), dtype(4.0)
    for i in range(iters):
        t_new = half * (one + np.sqrt(one + four * t * t))
        out[i] = (t - one) / t_new
        t = t_new
    return out


def fista_cs_single_coil(kspace_zf: np.ndarray, mask: np.ndarray, iters: int,
                         lam: float, alpha_dtype=np.float64) -> np.ndarray:
    """cs.rs:59-139.  ``kspace_zf`` is ``[..., ny, nx]`` (extra leading axes
    are independent problems, e.g. coils); ``mask`` broadcasts against it."""
    k = np.asarray(kspace_zf, dtype=np.complex128)
    m = np.asarray(mask, dtype=bool)
    ny, nx = k.shape[-2:]
    if m.shape[-2:] != (ny, nx):
        raise ValueError(f"CS: mask shape {m.shape} does not match kspace shape {(ny, nx)}")
    if ny % 2 or nx % 2:
        raise ValueError(f"CS: Ny ({ny}) and Nx ({nx}) must both be even for Haar wavelet")
    atb = centred_ifft2(np.where(m, k, 0))          # cs.rs:84-92
    x = atb.copy()                                   # cs.rs:95
    z = x.copy()
    for alpha in fista_alpha_table(iters, alpha_dtype):
        az = centred_fft2(z)                         # cs.rs:101-102
        az = np.where(m, az - k, 0)                  # cs.rs:103-111
        az = centred_ifft2(az)                       # cs.rs:112
        v = z - az                                   # cs.rs:114-119
        x_new = haar_inverse(soft_threshold_details(haar_forward(v), lam))  # cs.rs:120-122
        z = x_new + float(alpha) * (x_new - x)       # cs.rs:127-133
        x = x_new
    return x


# --------------------------------------------------------------------------
# coil.rs / crop.rs / strategy.rs epilogue
# --------------------------------------------------------------------------
def rss_combine(coil_images: np.ndarray) -> np.ndarray:
    """coil.rs:24-27 / strategy.rs:870-879: sqrt(sum_c |x_c|^2) over axis 0."""
    return np.sqrt(np.sum(np.abs(coil_images) ** 2, axis=0))


def center_crop_3d(vol: np.ndarray, target) -> np.ndarray:
    """crop.rs:13-27."""
    nz, ny, nx = vol.shape
    tz, ty, tx = target
    tz = max(min(tz, nz), 1)
    ty = max(min(ty, ny), 1)
    tx = max(min(tx, nx), 1)
    z0, y0, x0 = (nz - tz) // 2, (ny - ty) // 2, (nx - tx) // 2
    return vol[z0:z0 + tz, y0:y0 + ty, x0:x0 + tx].copy()


def maybe_crop(mag: np.ndarray, recon_matrix) -> np.ndarray:
    """strategy.rs:227-253 (IfftRss::maybe_crop); recon_matrix = (x, y, z)."""
    rx, ry, rz = recon_matrix
    nz, ny, nx = mag.shape
    tz = min(rz, nz) if rz >= 2 else nz
    ty = min(ry, ny) if ry >= 1 else ny
    tx = min(rx, nx) if rx >= 1 else nx
    if (tz, ty, tx) != (nz, ny, nx) and tx <= nx and ty <= ny and tz <= nz:
        return center_crop_3d(mag, (tz, ty, tx))
    return mag


# --------------------------------------------------------------------------
# fft.rs (kz decoupling and the odd-dimension fallback)
# --------------------------------------------------------------------------
def ifft_axis(a: np.ndarray, axis: int) -> np.ndarray:
    """fft.rs:59-84: inverse DFT along ``axis`` scaled by 1/n."""
    if a.shape[axis] < 2:
        return np.asarray(a, dtype=np.complex128).copy()
    return np.fft.ifft(np.asarray(a, dtype=np.complex128), axis=axis)


def ifft1_inplace(a: np.ndarray, axis: int) -> np.ndarray:
    """fft.rs:52-56: ifftshift -> IFFT(1/n) -> fftshift along one axis."""
    a = ifftshift_axis(np.asarray(a, dtype=np.complex128), axis)
    a = ifft_axis(a, axis)
    return fftshift_axis(a, axis)


def ifft2_inplace(a: np.ndarray, axes=(-2, -1)) -> np.ndarray:
    """fft.rs:19-29."""
    a1, a2 = axes
    a = ifftshift_axis(np.asarray(a, dtype=np.complex128), a1)
    a = ifftshift_axis(a, a2)
    a = ifft_axis(a, a1)
    a = ifft_axis(a, a2)
    a = fftshift_axis(a, a1)
    return fftshift_axis(a, a2)


# --------------------------------------------------------------------------
# prewhiten.rs
# --------------------------------------------------------------------------
def cholesky_lower(a: np.ndarray):
    """prewhiten.rs:148-179.  Returns None when a diagonal pivot's real part
    is not finite or <= 0 (the imaginary part of the pivot is ignored)."""
    n = a.shape[0]
    l = np.zeros((n, n), dtype=np.complex128)
    for i in range(n):
        diag = a[i, i] - np.sum(l[i, :i] * np.conj(l[i, :i]))
        d_re = diag.real
        if not np.isfinite(d_re) or d_re <= 0.0:
            return None
        l_ii = np.sqrt(d_re)
        l[i, i] = l_ii
        for j in range(i + 1, n):
            s = a[j, i] - np.sum(l[j, :i] * np.conj(l[i, :i]))
            l[j, i] = s * (1.0 / l_ii)
    return l


def invert_lower_triangular(l: np.ndarray, eps: float = float(np.finfo(np.float32).eps)):
    """prewhiten.rs:183-210: forward substitution per unit column; None when a
    diagonal entry has |re| < eps and |im| < eps."""
    n = l.shape[0]
    inv = np.zeros((n, n), dtype=np.complex128)
    for col in range(n):
        for i in range(n):
            s = (1.0 if i == col else 0.0) - np.sum(l[i, :i] * inv[:i, col])
            d = l[i, i]
            if abs(d.real) < eps and abs(d.imag) < eps:
                return None
            inv[i, col] = s / d
    return np.tril(inv)


def prewhitener_from_noise(noise_acqs):
    """prewhiten.rs:48-111.  ``noise_acqs`` is a list of ``[nc, ns]`` arrays.
    Returns W = L^-1 (lower triangular) or None (no samples / under-determined
    / not positive definite)."""
    if len(noise_acqs) == 0:
        return None
    nc = noise_acqs[0].shape[0]
    if nc == 0:
        return None
    total = sum(int(a.shape[1]) for a in noise_acqs)   # counts skipped scans too
    if total < nc:
        return None
    psi = np.zeros((nc, nc), dtype=np.complex128)
    for a in noise_acqs:
        if a.shape[0] != nc:
            continue
        s = np.asarray(a, dtype=np.complex128)
        psi += s @ np.conj(s.T)
    psi /= max(float(total) - 1.0, 1.0)
    l = cholesky_lower(psi)
    if l is None:
        return None
    return invert_lower_triangular(l)


def prewhiten_apply(w: np.ndarray, data: np.ndarray) -> np.ndarray:
    """prewhiten.rs:118-142: every sample column s -> W s.  ``data`` is
    ``[..., nc, ns]``; acquisitions with another channel count pass through."""
    if data.shape[-2] != w.shape[0]:
        return np.asarray(data).copy()
    return np.einsum("ij,...jn->...in", np.tril(w), np.asarray(data, dtype=np.complex128))


# --------------------------------------------------------------------------
# phasecorr.rs
# --------------------------------------------------------------------------
def phase_corrector_from_acqs(scans):
    """phasecorr.rs:61-129.  ``scans``: the phase-correction acquisitions in
    file order as (slice, segment, [nc, ns] array).  Bins by (slice, segment):
    the coil sum of each scan (channel order) is added to its bin in scan
    order; a scan whose ns differs from the bin's first scan is dropped, scans
    with no samples or channels are skipped.  Returns {(slice, segment):
    c(k) = conj(avg) / |avg|, or 1 where |avg| < 1e-20}."""
    bins = {}
    for sl, seg, d in scans:
        d = np.asarray(d, dtype=np.complex128)
        nc, ns = d.shape
        if ns == 0 or nc == 0:
            continue
        coil_sum = d.sum(axis=0)
        key = (int(sl), int(seg))
        if key not in bins:
            bins[key] = [np.zeros(ns, np.complex128), 0]
        if bins[key][0].shape[0] != ns:
            continue
        bins[key][0] = bins[key][0] + coil_sum
        bins[key][1] += 1
    out = {}
    for key, (total, count) in bins.items():
        avg = total * (1.0 / count)
        mag = np.abs(avg)
        out[key] = np.where(mag < 1e-20, 1.0 + 0j, np.conj(avg) / np.where(mag < 1e-20, 1.0, mag))
    return out


def phase_correct_apply(corr, data, slice_, segment):
    """phasecorr.rs:141-168: multiply the first min(ns, len(c)) samples of
    every channel by the phasor of (slice, segment), else of (65535, segment),
    else leave the line untouched."""
    c = corr.get((int(slice_), int(segment)))
    if c is None:
        c = corr.get((65535, int(segment)))
    d = np.asarray(data, dtype=np.complex128).copy()
    if c is None:
        return d
    n = min(d.shape[-1], c.shape[0])
    d[..., :n] *= c[:n]
    return d


# --------------------------------------------------------------------------
# oversampling.rs
# --------------------------------------------------------------------------
def oversampling_ratio(encoded_x: int, recon_x: int):
    """oversampling.rs:50-71: integer ratio <= 8, else None."""
    if recon_x == 0 or encoded_x <= recon_x or encoded_x % recon_x != 0:
        return None
    r = encoded_x // recon_x
    return None if r > 8 else r


def oversampling_apply(data: np.ndarray, encoded_x: int, recon_x: int) -> np.ndarray:
    """oversampling.rs:103-155 on ``[..., nc, ns]``: centred IFFT/enc ->
    crop [(enc-rec)/2, +rec) -> centred unnormalised FFT.  Acquisitions whose
    ns differs from enc pass through unchanged."""
    if data.shape[-1] != encoded_x:
        return np.asarray(data).copy()
    lane = np.asarray(data, dtype=np.complex128)
    lane = _rotate_left(lane, -1, (encoded_x + 1) // 2)
    lane = np.fft.ifft(lane, axis=-1)                    # unnormalised IFFT * 1/enc
    lane = _rotate_left(lane, -1, encoded_x // 2)
    start = (encoded_x - recon_x) // 2
    crop = lane[..., start:start + recon_x]
    crop = _rotate_left(crop, -1, (recon_x + 1) // 2)
    crop = np.fft.fft(crop, axis=-1)
    return _rotate_left(crop, -1, recon_x // 2)


# --------------------------------------------------------------------------
# strategy.rs:782-891 (CsRss::reconstruct after the read pass)
# --------------------------------------------------------------------------
def csrss_from_kspace(kspace: np.ndarray, mask: np.ndarray, iters: int, lam: float,
                      three_d: bool = False, recon_matrix=None,
                      return_coils: bool = False, workers: int = 1):
    """strategy.rs:817-891 on placed k-space ``[nc, nz, ny, nx]`` and
    ``mask [nz, ny, nx]``: optional kz decoupling, odd-dim fallback to
    IFFT+RSS, per-slice per-coil FISTA, RSS, optional crop.  ``workers`` > 1
    solves the coils of a slice on that many threads (the coil solves are
    independent, strategy.rs:850-869; the results are the same)."""
    k = np.asarray(kspace, dtype=np.complex128)
    if three_d:
        k = ifft1_inplace(k, 1)                          # strategy.rs:824-827
    nc, nz, ny, nx = k.shape
    if ny % 2 or nx % 2:                                 # strategy.rs:829-842
        mag = rss_combine(ifft2_inplace(k, (2, 3)))
        return maybe_crop(mag, recon_matrix) if recon_matrix is not None else mag
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    coils = np.zeros_like(k) if return_coils else None
    pool = None
    if workers > 1 and nc > 1:
        from concurrent.futures import ThreadPoolExecutor
        pool = ThreadPoolExecutor(min(workers, nc))
    for kz in range(nz):
        if pool is not None:
            x = np.stack(list(pool.map(lambda c: fista_cs_single_coil(k[c, kz], mask[kz], iters, lam), range(nc))))
        else:
            x = fista_cs_single_coil(k[:, kz], mask[kz], iters, lam)
        out[kz] = rss_combine(x)
        if return_coils:
            coils[:, kz] = x
    if pool is not None:
        pool.shutdown()
    if recon_matrix is not None:
        out = maybe_crop(out, recon_matrix)
    return (out, coils) if return_coils else out


def nrmse(a: np.ndarray, ref: np.ndarray) -> float:
    """||a - ref||_2 / ||ref||_2 (the accuracy metric of the benchmarks)."""
    ref = np.asarray(ref)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((np.asarray(a) - ref).ravel()) / (den if den > 0 else 1.0))
