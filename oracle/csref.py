"""ctypes wrapper of ``oracle/libcsref.so`` (the FP32 C restatement).

Test infrastructure only.  Arrays are numpy complex64 (interleaved re/im
float pairs, the layout of the reference's ``Complex32``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcsref.so")
_lib = None

_f = ctypes.POINTER(ctypes.c_float)
_u8 = ctypes.POINTER(ctypes.c_uint8)


def build() -> str:
    """Compile the restatement with oracle/Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
                os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "cs_ref.c"))):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.csref_fft_1d.argtypes = [_f, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.csref_centred_fft2.argtypes = [_f, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.csref_haar_forward.argtypes = [_f, _f, ctypes.c_int, ctypes.c_int]
        L.csref_haar_inverse.argtypes = [_f, _f, ctypes.c_int, ctypes.c_int]
        L.csref_soft_threshold_details.argtypes = [_f, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.csref_fista_cs_single_coil.argtypes = [_f, _u8, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, _f]
        L.csref_csrss.argtypes = [_f, _u8, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_float, ctypes.c_int, _f, _f]
        L.csref_prewhiten_fit.argtypes = [_f, ctypes.c_int, ctypes.c_long, _f]
        L.csref_prewhiten_apply.argtypes = [_f, _f, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.csref_os_apply.argtypes = [_f, _f, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.csref_ifft1_axis.argtypes = [_f, ctypes.c_long, ctypes.c_int, ctypes.c_long]
        L.csref_sense_unfold.argtypes = [_f, _f, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_float, _f, _f]
        _lib = L
    return _lib


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex64)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_f)


def fft_1d(x, inverse=False) -> np.ndarray:
    """Unnormalised DFT along the last axis."""
    a = _c64(x).copy()
    n = a.shape[-1]
    lib().csref_fft_1d(_fp(a), n, a.size // max(n, 1), int(inverse))
    return a


def centred_fft2(x, inverse=False) -> np.ndarray:
    a = _c64(x).copy()
    ny, nx = a.shape[-2:]
    lib().csref_centred_fft2(_fp(a), ny, nx, a.size // (ny * nx), int(inverse))
    return a


def haar_forward(x) -> np.ndarray:
    a = _c64(x)
    out = np.empty_like(a)
    rc = lib().csref_haar_forward(_fp(a), _fp(out), a.shape[0], a.shape[1])
    if rc:
        raise ValueError("Haar: dims must be even")
    return out


def haar_inverse(x) -> np.ndarray:
    a = _c64(x)
    out = np.empty_like(a)
    rc = lib().csref_haar_inverse(_fp(a), _fp(out), a.shape[0], a.shape[1])
    if rc:
        raise ValueError("Haar: dims must be even")
    return out


def soft_threshold_details(x, lam) -> np.ndarray:
    a = _c64(x).copy()
    lib().csref_soft_threshold_details(_fp(a), a.shape[0], a.shape[1], float(lam))
    return a


def fista_cs_single_coil(kspace_zf, mask, iters, lam) -> np.ndarray:
    k = _c64(kspace_zf)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    ny, nx = k.shape
    out = np.empty_like(k)
    rc = lib().csref_fista_cs_single_coil(_fp(k), m.ctypes.data_as(_u8), ny, nx, int(iters),
                                          float(lam), _fp(out))
    if rc:
        raise ValueError(f"CS: Ny ({ny}) and Nx ({nx}) must both be even for Haar wavelet")
    return out


def csrss(kspace, mask, iters, lam, nthreads=1, return_coils=False):
    """Per-slice per-coil FISTA + f32 RSS; kspace [nc,nz,ny,nx], mask [nz,ny,nx]."""
    k = _c64(kspace)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    nc, nz, ny, nx = k.shape
    out = np.empty((nz, ny, nx), dtype=np.float32)
    coils = np.empty_like(k) if return_coils else None
    rc = lib().csref_csrss(_fp(k), m.ctypes.data_as(_u8), nc, nz, ny, nx, int(iters), float(lam),
                           int(nthreads), out.ctypes.data_as(_f),
                           _fp(coils) if coils is not None else None)
    if rc:
        raise ValueError("CS: odd dimensions")
    return (out, coils) if return_coils else out


def prewhiten_fit(noise):
    """noise [nc, ns] -> W [nc, nc] or None (skipped)."""
    a = _c64(noise)
    nc, ns = a.shape
    w = np.zeros((nc, nc), dtype=np.complex64)
    rc = lib().csref_prewhiten_fit(_fp(a), nc, ns, _fp(w))
    return None if rc else w


def prewhiten_apply(w, data) -> np.ndarray:
    """data [..., nc, ns]."""
    a = _c64(data).copy()
    nc, ns = a.shape[-2:]
    lib().csref_prewhiten_apply(_fp(_c64(w)), _fp(a), a.size // (nc * ns), nc, ns)
    return a


def oversampling_apply(data, enc, rec) -> np.ndarray:
    a = _c64(data)
    nc = a.shape[-2]
    nacq = a.size // (nc * enc)
    out = np.empty(a.shape[:-1] + (rec,), dtype=np.complex64)
    rc = lib().csref_os_apply(_fp(a), _fp(out), nacq, nc, enc, rec)
    if rc:
        raise ValueError("invalid oversampling ratio")
    return out


def ifft1_axis(data, axis) -> np.ndarray:
    a = _c64(data).copy()
    n = a.shape[axis]
    outer = int(np.prod(a.shape[:axis]))
    inner = int(np.prod(a.shape[axis + 1:]))
    lib().csref_ifft1_axis(_fp(a), outer, n, inner)
    return a


def sense_unfold(aliased, maps, r, ridge, gfactor=False):
    """sense.rs:64-252 in f32: (unfolded [ny, nx] complex64, g-factor [ny, nx]
    float32 or None)."""
    a, m = _c64(aliased), _c64(maps)
    nc, ny, nx = a.shape
    out = np.zeros((ny, nx), np.complex64)
    g = np.zeros((ny, nx), np.float32) if gfactor else None
    rc = lib().csref_sense_unfold(_fp(a), _fp(m), nc, ny, nx, int(r), float(ridge), _fp(out),
                                  g.ctypes.data_as(_f) if g is not None else None)
    if rc:
        raise ValueError("SENSE: bad R")
    return out, g
