"""FP64 oracle of the SENSE extension mode -- test infrastructure only.

The reference's ``cs`` strategy is per-coil (strategy.rs:736-892; cs.rs:23-26
names SENSE-CS as a follow-up).  The extension mode solves one image per
slice with coil sensitivity maps:

    min_x  1/2 sum_c || M F (S_c x) - y_c ||^2  +  lambda || W x ||_1

by FISTA with step 1/L, L = ||A||^2 from an FP64 power iteration, warm start
x0 = z0 = A^H y, the reference's Haar prox (threshold lambda / L, LL band
untouched) and momentum (cs.rs:99-137).  Maps: Walsh's method
(sensitivity.rs:37-142) on the low-resolution coil images of the ACS block
(the longest run of sampled ky rows, grappa.rs:50-87; images as in
strategy.rs:658-671), then normalised to unit root-sum-of-squares.
"""
from __future__ import annotations

import numpy as np

from oracle import cs_fp64 as o64


def acs_rows(rows: np.ndarray):
    """grappa.rs:50-87: the longest run of consecutive sampled rows (first
    longest wins); None when fewer than 4 rows are sampled."""
    s = np.flatnonzero(np.asarray(rows, bool))
    if s.size < 4:
        return None
    best_start, best_len = 0, 0
    cur_start, cur_len = int(s[0]), 1
    for a, b in zip(s[:-1], s[1:]):
        if b == a + 1:
            cur_len += 1
        else:
            if cur_len > best_len:
                best_len, best_start = cur_len, cur_start
            cur_start, cur_len = int(b), 1
    if cur_len > best_len:
        best_len, best_start = cur_len, cur_start
    return best_start, best_start + best_len


def lowres_images(kspace: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """strategy.rs:658-669: k-space of the ACS rows only, centred IFFT2 (1/N)."""
    a0, a1 = acs_rows(rows)
    k = np.zeros_like(np.asarray(kspace, np.complex128))
    k[:, a0:a1, :] = kspace[:, a0:a1, :]
    return o64.ifft2_inplace(k, (1, 2))


def walsh_maps(imgs: np.ndarray, window: int = 3, power_iters: int = 6) -> np.ndarray:
    """sensitivity.rs:37-142 (per pixel, loops over the clipped window)."""
    nc, ny, nx = imgs.shape
    out = np.zeros((nc, ny, nx), np.complex128)
    s = imgs.reshape(nc, -1)
    for y in range(ny):
        y0, y1 = max(y - window, 0), min(y + window + 1, ny)
        for x in range(nx):
            x0, x1 = max(x - window, 0), min(x + window + 1, nx)
            blk = imgs[:, y0:y1, x0:x1].reshape(nc, -1)
            r = blk @ np.conj(blk.T)                       # sum s s^H
            v = imgs[:, y, x].astype(np.complex128)
            nrm0 = np.sum(np.abs(v) ** 2)
            if nrm0 == 0:
                v = np.zeros(nc, np.complex128)
                v[0] = 1.0
            else:
                v = v / np.sqrt(nrm0)
            lam = 0.0
            for _ in range(power_iters):
                w = r @ v
                nrm = np.sqrt(np.sum(np.abs(w) ** 2))
                if nrm < 1e-20:
                    break
                v = w / nrm
                lam = nrm
            m = np.abs(v)
            imax = int(np.argmax(m)) if m.max() > 0 else 0
            if m[imax] > 0:
                v = v * (np.conj(v[imax]) / m[imax])
            out[:, y, x] = v * np.sqrt(lam)
    del s
    return out


def normalise_maps(maps: np.ndarray) -> np.ndarray:
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(rss > 0, maps / np.where(rss > 0, rss, 1), 0)


def _normal_op(maps, mask, v):
    """A^H A v = sum_c S_c^* F^H M F (S_c v)."""
    u = o64.centred_fft2(maps * v[None])
    u = np.where(mask[None], u, 0)
    return np.sum(np.conj(maps) * o64.centred_ifft2(u), axis=0)


def lipschitz(maps: np.ndarray, mask: np.ndarray, iters: int = 30, seed: int = 0) -> float:
    """||A||^2 by power iteration on A^H A (FP64), starting from all-ones."""
    ny, nx = mask.shape
    v = np.ones((ny, nx), np.complex128) / np.sqrt(ny * nx)
    lam = 0.0
    for _ in range(iters):
        w = _normal_op(maps, mask, v)
        lam = float(np.sqrt(np.sum(np.abs(w) ** 2)))
        if lam == 0:
            return 0.0
        v = w / lam
    return lam


def sense_fista(kspace, maps, mask, iters, lam, L):
    """cs.rs:59-139 structure with the SENSE operator and step 1/L."""
    k = np.asarray(kspace, np.complex128)
    m = np.asarray(mask, bool)
    atb = np.sum(np.conj(maps) * o64.centred_ifft2(np.where(m[None], k, 0)), axis=0)
    x = atb.copy()
    z = x.copy()
    for alpha in o64.fista_alpha_table(iters):
        g = _normal_op(maps, m, z) - atb
        v = z - g / L
        x_new = o64.haar_inverse(o64.soft_threshold_details(o64.haar_forward(v), lam / L))
        z = x_new + float(alpha) * (x_new - x)
        x = x_new
    return x


def sense_unfold_1d(aliased, maps, r: int, ridge: float, gfactor: bool = False):
    """sense.rs:64-252 in FP64: rho = (C^H C + ridge I)^-1 C^H (R a) per
    reduced voxel through the prewhiten.rs Cholesky and triangular inverse;
    voxels whose factorisation fails stay zero.  Returns (unfolded [ny, nx],
    g-factor [ny, nx] or None)."""
    a = np.asarray(aliased, dtype=np.complex128)
    m = np.asarray(maps, dtype=np.complex128)
    nc, ny, nx = a.shape
    if r < 1 or ny % r:
        raise ValueError("SENSE: bad R")
    nyr = ny // r
    out = np.zeros((ny, nx), np.complex128)
    g = np.zeros((ny, nx), np.float64) if gfactor else None
    for x in range(nx):
        for y0 in range(nyr):
            C = m[:, y0 + nyr * np.arange(r), x]                 # [nc, r]
            chc = C.conj().T @ C + ridge * np.eye(r)
            rhs = (C.conj().T @ a[:, y0, x]) * r
            low = o64.cholesky_lower(chc)
            if low is None:
                continue
            inv = o64.invert_lower_triangular(low)
            if inv is None:
                continue
            rho = inv.conj().T @ (inv @ rhs)
            out[y0 + nyr * np.arange(r), x] = rho
            if g is not None:
                inv_diag = np.sum(np.abs(inv) ** 2, axis=0)
                g[y0 + nyr * np.arange(r), x] = np.sqrt(np.maximum(inv_diag * np.maximum(chc.diagonal().real, 0), 0))
    return out, g
