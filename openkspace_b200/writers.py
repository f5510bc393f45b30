"""Output writers of the reconstruction (openkspace-cli/src/main.rs:1033-1153)
over the C-ABI: NIfTI-1 volumes, and 8-bit PNG slices windowed by percentiles
(or linearly) on the device.

``write_png_windowed`` / ``write_png_linear`` take the slice as a device array
(DeviceArray [ny, nx] float32) or a host array; the percentiles come from the
device's radix select (okscuda_percentile) and the byte mapping from
okscuda_window_u8, so only the 8-bit image crosses to the host.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import OksError

FLT_EPSILON = np.float32(np.finfo(np.float32).eps)


def write_nifti_volume(vol, path: str):
    """main.rs:1033-1074: vol [nz, ny, nx] float32 (host array or DeviceArray)."""
    v = vol.to_host() if hasattr(vol, "to_host") else np.ascontiguousarray(vol, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    nz, ny, nx = v.shape
    rc = _lib.load().okscuda_write_nifti(v.ctypes.data, nz, ny, nx, os.fsencode(path))
    if rc != 0:
        raise OksError(rc, f"writing {path}")


def percentile(ctx, d_vals, pct: float) -> float:
    """main.rs:1147-1153 on the device (exact order statistic)."""
    d, _ = ctx._dev(d_vals, np.float32)
    out = ctypes.c_float()
    ctx.check(ctx.lib.okscuda_percentile(ctx.handle, d.ptr, d.size, float(pct), ctypes.byref(out)))
    return float(out.value)


def window_u8(ctx, d_img, lo: float, hi: float, gamma: bool) -> np.ndarray:
    """main.rs:1095-1140 pixel mapping on the device; returns the bytes."""
    d, _ = ctx._dev(d_img, np.float32)
    o = ctx.empty(d.shape, np.uint8)
    ctx.check(ctx.lib.okscuda_window_u8(ctx.handle, d.ptr, d.size, float(lo), float(hi), int(gamma), o.ptr))
    return o.to_host()


def write_png(gray: np.ndarray, path: str):
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    h, w = g.shape
    rc = _lib.load().okscuda_write_png(g.ctypes.data, w, h, os.fsencode(path))
    if rc != 0:
        raise OksError(rc, f"writing {path}")


def write_png_windowed(ctx, img, path: str, pct_low: float = 1.0, pct_high: float = 99.5) -> np.ndarray:
    """main.rs:1112-1140: window [percentile(pct_low), percentile(pct_high)],
    gamma 0.9.  Returns the 8-bit image written."""
    d, _ = ctx._dev(img, np.float32)
    lo = np.float32(percentile(ctx, d, pct_low))
    hi = max(np.float32(percentile(ctx, d, pct_high)), np.float32(lo + FLT_EPSILON))
    g = window_u8(ctx, d, lo, hi, True)
    write_png(g, path)
    return g


def write_png_linear(ctx, img, path: str, lo: float, hi: float) -> np.ndarray:
    """main.rs:1095-1110: fixed window [lo, hi]."""
    g = window_u8(ctx, img, lo, hi, False)
    write_png(g, path)
    return g
