"""Restatement of the reference's output writers (test infrastructure only):
openkspace-cli/src/main.rs:1095-1153 -- percentile(), the 8-bit pixel maps of
write_png_linear / write_png_windowed -- and a reader of the NIfTI-1 header
fields main.rs:1033-1074 writes.  f32 arithmetic throughout, in the
reference's order."""
from __future__ import annotations

import struct

import numpy as np

EPS32 = np.float32(np.finfo(np.float32).eps)


def _round_half_away(x):
    """f32 round() of Rust / C roundf for x >= 0: floor, plus one when the
    (exact) fraction is at least one half."""
    x = np.asarray(x, dtype=np.float32)
    f = np.floor(x)
    return np.where((x - f) >= np.float32(0.5), f + np.float32(1.0), f)


def percentile(values, pct: float) -> np.float32:
    """main.rs:1147-1153 on the ascending sort of ``values``."""
    s = np.sort(np.asarray(values, dtype=np.float32).ravel())
    if s.size == 0:
        return np.float32(0.0)
    fk = np.float32(np.float32(pct) / np.float32(100.0)) * np.float32(s.size - 1)
    k = int(max(float(_round_half_away(max(fk, np.float32(0.0)))), 0.0))   # `as usize` saturates at 0
    return s[min(k, s.size - 1)]


def window_u8(img, lo, hi, gamma: bool) -> np.ndarray:
    """main.rs:1097-1107 (gamma False) and main.rs:1124-1136 (gamma True)."""
    lo, hi = np.float32(lo), np.float32(hi)
    hi = max(hi, np.float32(lo + EPS32))
    v = np.asarray(img, dtype=np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        norm = np.clip((v - lo) / np.float32(hi - lo), np.float32(0.0), np.float32(1.0)).astype(np.float32)
        g = np.power(norm, np.float32(0.9)).astype(np.float32) if gamma else norm
        x = (g * np.float32(255.0)).astype(np.float32)
    r = _round_half_away(np.where(np.isnan(x), np.float32(0.0), x))
    return r.astype(np.uint8)


def png_windowed(img, pct_low, pct_high) -> np.ndarray:
    """main.rs:1112-1140: the bytes write_png_windowed saves."""
    lo = percentile(img, pct_low)
    hi = max(percentile(img, pct_high), np.float32(lo + EPS32))
    return window_u8(img, lo, hi, True)


def nifti_header(raw: bytes) -> dict:
    """The fields main.rs:1033-1074 sets, read back (little-endian)."""
    return {"sizeof_hdr": struct.unpack_from("<i", raw, 0)[0],
            "dim": struct.unpack_from("<8h", raw, 40),
            "datatype": struct.unpack_from("<h", raw, 70)[0],
            "bitpix": struct.unpack_from("<h", raw, 72)[0],
            "pixdim": struct.unpack_from("<8f", raw, 76),
            "vox_offset": struct.unpack_from("<f", raw, 108)[0],
            "scl_slope": struct.unpack_from("<f", raw, 112)[0],
            "magic": raw[344:348]}
