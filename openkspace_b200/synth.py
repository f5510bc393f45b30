"""Seeded synthetic MRI inputs for the FISTA-CS workloads.

No public dataset items are used: every array is drawn from numpy's PCG64
with seed ``1000 * workload + slice``.

* phantom: 10 random ellipses (centres, axes, angles uniform in the FOV,
  intensities U(0.1, 1)) times a smooth random phase exp(i * low-order
  polynomial);
* coils: Gaussian bumps placed round the FOV, normalised to unit
  root-sum-of-squares per pixel;
* k-space: y_c = F(S_c * rho) with the centred unitary 2-D FFT of the
  reference (cs.rs:141-178), plus complex Gaussian noise of sigma
  1e-3 * max|y| (optionally correlated across channels);
* masks: ky-only (constant along kx): exactly round(ny / R) rows including a
  fully sampled centre block.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.fft as sfft


def _centred_fft2(a: np.ndarray) -> np.ndarray:
    ny, nx = a.shape[-2:]
    a = np.fft.ifftshift(a, axes=(-2, -1)) if (ny % 2 == 0 and nx % 2 == 0) else \
        np.roll(np.roll(a, -((ny + 1) // 2), -2), -((nx + 1) // 2), -1)
    a = sfft.fft2(a, axes=(-2, -1), workers=-1)
    a = np.roll(np.roll(a, -(ny // 2), -2), -(nx // 2), -1)
    return a / np.sqrt(float(ny) * nx)


def ellipse_phantom(ny: int, nx: int, rng: np.random.Generator, n_ellipses: int = 10,
                    obj_nx: int | None = None) -> np.ndarray:
    """Complex phantom [ny, nx]; the object lies in the central ``obj_nx``
    columns (all of them by default; fewer for a readout-oversampled FOV)."""
    obj_nx = nx if obj_nx is None else obj_nx
    yy, xx = np.meshgrid(np.linspace(-1, 1, ny, endpoint=False),
                         np.linspace(-1, 1, obj_nx, endpoint=False), indexing="ij")
    img = np.zeros((ny, obj_nx))
    for _ in range(n_ellipses):
        cy, cx = rng.uniform(-0.6, 0.6, 2)
        ay, ax = rng.uniform(0.08, 0.5, 2)
        th = rng.uniform(0, np.pi)
        val = rng.uniform(0.1, 1.0)
        c, s = np.cos(th), np.sin(th)
        u = ((xx - cx) * c + (yy - cy) * s) / ax
        v = (-(xx - cx) * s + (yy - cy) * c) / ay
        img[u * u + v * v <= 1.0] += val
    coef = rng.uniform(-1.0, 1.0, 6)
    phase = (coef[0] + coef[1] * yy + coef[2] * xx + 0.5 * coef[3] * yy * yy
             + 0.5 * coef[4] * xx * xx + 0.5 * coef[5] * xx * yy)
    obj = img * np.exp(1j * np.pi * 0.5 * phase)
    if obj_nx == nx:
        return obj
    out = np.zeros((ny, nx), dtype=np.complex128)
    x0 = (nx - obj_nx) // 2
    out[:, x0:x0 + obj_nx] = obj
    return out


def coil_maps(nc: int, ny: int, nx: int, rng: np.random.Generator) -> np.ndarray:
    """Gaussian-bump sensitivities round the FOV, unit RSS per pixel."""
    yy, xx = np.meshgrid(np.linspace(-1, 1, ny, endpoint=False),
                         np.linspace(-1, 1, nx, endpoint=False), indexing="ij")
    maps = np.empty((nc, ny, nx), dtype=np.complex128)
    for c in range(nc):
        ang = 2 * np.pi * c / nc + rng.uniform(-0.2, 0.2)
        r = rng.uniform(0.9, 1.3)
        cy, cx = r * np.sin(ang), r * np.cos(ang)
        w = rng.uniform(0.6, 1.0)
        mag = np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * w * w))
        ph = rng.uniform(-np.pi, np.pi) + 0.5 * rng.uniform(-1, 1) * (yy + xx)
        maps[c] = mag * np.exp(1j * ph)
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    return maps / rss


def ky_mask(ny: int, accel: float, n_centre: int, rng: np.random.Generator) -> np.ndarray:
    """Boolean [ny] row mask: a centred block of ``n_centre`` rows plus random
    rows, round(ny / accel) rows in total."""
    total = max(int(round(ny / accel)), min(n_centre, ny))
    m = np.zeros(ny, dtype=bool)
    c0 = ny // 2 - n_centre // 2
    m[max(c0, 0):min(c0 + n_centre, ny)] = True
    rest = np.flatnonzero(~m)
    extra = total - int(m.sum())
    if extra > 0:
        m[rng.choice(rest, size=min(extra, rest.size), replace=False)] = True
    return m


def noise_covariance(nc: int, cond: float, rng: np.random.Generator) -> np.ndarray:
    """Hermitian positive-definite Psi = Q diag(d) Q^H, d log-spaced [1, cond]."""
    g = rng.standard_normal((nc, nc)) + 1j * rng.standard_normal((nc, nc))
    q, r = np.linalg.qr(g)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    d = np.logspace(0, np.log10(cond), nc)
    return (q * d) @ np.conj(q.T)


@dataclasses.dataclass
class Slice:
    kspace: np.ndarray      # [nc, ny, nx] complex64, zero-filled (rows outside mask = 0)
    mask_rows: np.ndarray   # [ny] bool
    truth: np.ndarray       # [ny, nx] complex128 phantom

    @property
    def mask2d(self) -> np.ndarray:
        return np.repeat(self.mask_rows[:, None], self.kspace.shape[-1], axis=1)


def make_slice(ny: int, nx: int, nc: int, accel: float, n_centre: int, seed: int,
               noise_rel: float = 1e-3) -> Slice:
    rng = np.random.Generator(np.random.PCG64(seed))
    rho = ellipse_phantom(ny, nx, rng)
    maps = coil_maps(nc, ny, nx, rng)
    k = _centred_fft2(maps * rho)
    sigma = noise_rel * np.abs(k).max()
    k = k + sigma * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)) / np.sqrt(2)
    m = ky_mask(ny, accel, n_centre, rng)
    k[:, ~m, :] = 0
    return Slice(k.astype(np.complex64), m, rho)


# --------------------------------------------------------------------------
# named workloads (sizes of the benchmark configurations)
# --------------------------------------------------------------------------
def plain_slice(seed_slice: int = 0) -> Slice:
    """8 coils, 256 x 256, R = 4 + 24 centre lines (lambda 0.01, 50 iters)."""
    return make_slice(256, 256, 8, 4.0, 24, 1000 * 0 + seed_slice)


@dataclasses.dataclass
class OversampledVolume:
    """Readout-oversampled multi-slice acquisition, as raw lines."""
    lines: np.ndarray        # [nz, n_lines, nc, enc_x] complex64 (sampled ky lines only)
    ky_index: np.ndarray     # [nz, n_lines] int32 row index of every line
    mask_rows: np.ndarray    # [nz, ny] bool
    noise: np.ndarray        # [nc, n_noise] complex64 noise-calibration samples
    psi: np.ndarray          # true noise covariance [nc, nc]
    ny: int
    enc_x: int
    rec_x: int

    def zero_filled(self) -> np.ndarray:
        """[nc, nz, ny, enc_x] zero-filled k-space (placement of the lines)."""
        nz, nl, nc, ex = self.lines.shape
        k = np.zeros((nc, nz, self.ny, ex), dtype=np.complex64)
        for z in range(nz):
            k[:, z, self.ky_index[z]] = np.transpose(self.lines[z], (1, 0, 2))
        return k


def oversampled_volume(nz: int = 36, nc: int = 15, ny: int = 368, enc_x: int = 640,
                       rec_x: int = 320, accel: float = 4.0, centre_frac: float = 0.08,
                       n_noise: int = 256, cond: float = 50.0, workload: int = 1,
                       noise_rel: float = 1e-3) -> OversampledVolume:
    """15 coils, 640 (readout, 2x oversampled) x 368 ky, 36 slices, R = 4 with
    an 8 % centre, noise correlated across channels (condition number 50),
    256 noise-calibration samples per coil."""
    rng0 = np.random.Generator(np.random.PCG64(1000 * workload + 999))
    psi = noise_covariance(nc, cond, rng0)
    evals, evecs = np.linalg.eigh(psi)
    sqrt_psi = (evecs * np.sqrt(np.maximum(evals, 0))) @ np.conj(evecs.T)
    n_centre = int(round(centre_frac * ny))
    n_lines = max(int(round(ny / accel)), n_centre)
    lines = np.zeros((nz, n_lines, nc, enc_x), dtype=np.complex64)
    ky_idx = np.zeros((nz, n_lines), dtype=np.int32)
    masks = np.zeros((nz, ny), dtype=bool)
    sigma0 = None
    for z in range(nz):
        rng = np.random.Generator(np.random.PCG64(1000 * workload + z))
        rho = ellipse_phantom(ny, enc_x, rng, obj_nx=rec_x)
        maps = coil_maps(nc, ny, enc_x, rng)
        m = ky_mask(ny, accel, n_centre, rng)
        rows = np.flatnonzero(m)
        k = _centred_fft2(maps * rho)[:, rows, :]           # [nc, n_lines, enc_x]
        if sigma0 is None:
            sigma0 = noise_rel * np.abs(k).max() / np.sqrt(np.mean(evals))
        wn = (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)) / np.sqrt(2)
        k = k + sigma0 * np.einsum("ij,jln->iln", sqrt_psi, wn)
        lines[z] = np.transpose(k, (1, 0, 2)).astype(np.complex64)
        ky_idx[z] = rows
        masks[z] = m
    wn = (rng0.standard_normal((nc, n_noise)) + 1j * rng0.standard_normal((nc, n_noise))) / np.sqrt(2)
    noise = (sigma0 * (sqrt_psi @ wn)).astype(np.complex64)
    return OversampledVolume(lines, ky_idx, masks, noise, psi, ny, enc_x, rec_x)


BATCHED_SIZES = ((256, 256), (320, 320), (384, 384), (368, 640))


@dataclasses.dataclass
class SliceRequest:
    kspace: np.ndarray     # [nc, ny, nx] complex64
    mask_rows: np.ndarray  # [ny] bool
    iters: int
    lam: float


def uneven_requests(n: int = 64, workload: int = 2, lam: float = 0.01,
                    sizes=BATCHED_SIZES, coil_range=(8, 32), accels=(2, 3, 4, 6),
                    iter_range=(30, 150)) -> list[SliceRequest]:
    """Slices of uneven matrix size, coil count, R and iteration count."""
    rng = np.random.Generator(np.random.PCG64(1000 * workload + 777))
    out = []
    for s in range(n):
        ny, nx = sizes[rng.integers(len(sizes))]
        nc = int(rng.integers(coil_range[0], coil_range[1] + 1))
        r = float(accels[rng.integers(len(accels))])
        iters = int(rng.integers(iter_range[0], iter_range[1] + 1))
        sl = make_slice(ny, nx, nc, r, 24, 1000 * workload + s)
        out.append(SliceRequest(sl.kspace, sl.mask_rows, iters, lam))
    return out


def volume_3d(nc: int = 32, nz: int = 192, ny: int = 256, nx: int = 256, accel: float = 6.0,
              n_centre: int = 24, workload: int = 4, noise_rel: float = 1e-3):
    """3-D Cartesian k-space [nc, nz, ny, nx] (complex64) with one ky-only
    mask shared by every kz; returns (kspace, mask_rows[ny])."""
    rng = np.random.Generator(np.random.PCG64(1000 * workload))
    m = ky_mask(ny, accel, n_centre, rng)
    zz, yy, xx = np.meshgrid(np.linspace(-1, 1, nz, endpoint=False),
                             np.linspace(-1, 1, ny, endpoint=False),
                             np.linspace(-1, 1, nx, endpoint=False), indexing="ij")
    vol = np.zeros((nz, ny, nx), dtype=np.complex64)
    for _ in range(10):
        c = rng.uniform(-0.5, 0.5, 3)
        a = rng.uniform(0.1, 0.5, 3)
        val = rng.uniform(0.1, 1.0)
        vol[((zz - c[0]) / a[0]) ** 2 + ((yy - c[1]) / a[1]) ** 2 + ((xx - c[2]) / a[2]) ** 2 <= 1] += val
    del zz, yy, xx
    maps2 = coil_maps(nc, ny, nx, rng).astype(np.complex64)
    k = np.empty((nc, nz, ny, nx), dtype=np.complex64)
    for c in range(nc):
        img = vol * maps2[c][None]
        kk = sfft.fftshift(sfft.fftn(sfft.ifftshift(img), workers=-1)) / np.sqrt(float(nz * ny * nx))
        k[c] = kk.astype(np.complex64)
    sigma = noise_rel * float(np.abs(k).max())
    k += (sigma * (rng.standard_normal(k.shape, dtype=np.float32)
                   + 1j * rng.standard_normal(k.shape, dtype=np.float32)) / np.sqrt(2)).astype(np.complex64)
    k[:, :, ~m, :] = 0
    return k, m
