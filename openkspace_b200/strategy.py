"""Drop-in mirror of the reference's ``CsRss`` strategy (strategy.rs:736-892).

``AcquisitionSet`` stands in for ``IsmrmrdFile`` as the ``cs`` path sees it
(acquisition headers + samples + the encoding block of the XML header);
``CsRss`` has the reference's public fields and defaults, ``name() == "cs"``,
and ``reconstruct()`` returns an ``ImageVolume`` (magnitude [slice, y, x]).
All the work runs in ``libokscuda.so`` (okscuda_csrss_reconstruct).
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from ._lib import OksError

# ISMRMRD acquisition flag bits (acquisition.rs:69-95): 1 << (position - 1)
ACQ_IS_NOISE_MEASUREMENT = 1 << 18
ACQ_IS_REVERSE = 1 << 21
ACQ_IS_NAVIGATION_DATA = 1 << 22
ACQ_IS_PHASECORR_DATA = 1 << 23

# okscuda_acq_header (include/okscuda.h)
HEADER_DTYPE = np.dtype([("flags", "<u8"), ("number_of_samples", "<u2"), ("active_channels", "<u2"),
                         ("discard_pre", "<u2"), ("discard_post", "<u2"), ("center_sample", "<u2"),
                         ("kspace_encode_step_1", "<u2"), ("kspace_encode_step_2", "<u2"), ("slice", "<u2"),
                         ("segment", "<u2"), ("data_offset", "<i8")], align=True)
assert HEADER_DTYPE.itemsize == 40 and HEADER_DTYPE.fields["data_offset"][1] == 32


class _AcqSet(ctypes.Structure):
    _fields_ = [("n_acq", ctypes.c_longlong), ("headers", ctypes.c_void_p), ("data", ctypes.c_void_p),
                ("data_len", ctypes.c_longlong), ("data_on_device", ctypes.c_int),
                ("enc_x", ctypes.c_int), ("enc_y", ctypes.c_int), ("enc_z", ctypes.c_int),
                ("rec_x", ctypes.c_int), ("rec_y", ctypes.c_int), ("rec_z", ctypes.c_int),
                ("ky_center", ctypes.c_int), ("kz_center", ctypes.c_int)]


class _Cfg(ctypes.Structure):
    _fields_ = [("remove_oversampling", ctypes.c_int), ("prewhiten", ctypes.c_int),
                ("phase_correct", ctypes.c_int), ("iters", ctypes.c_int), ("lambda_", ctypes.c_float),
                ("fft_mode", ctypes.c_int), ("crop_to_recon_matrix", ctypes.c_int)]


@dataclasses.dataclass
class AcquisitionSet:
    """Acquisitions in file order: ``headers`` (HEADER_DTYPE) and one flat
    complex64 ``data`` array (each acquisition [channels, samples] at its
    ``data_offset``), plus encoded / recon matrix and the ky/kz centre."""
    headers: np.ndarray
    data: np.ndarray
    encoded: tuple          # (x, y, z)
    recon: tuple            # (x, y, z)
    ky_center: int
    kz_center: int = 0

    def acquisition(self, i: int) -> np.ndarray:
        h = self.headers[i]
        n = int(h["active_channels"]) * int(h["number_of_samples"])
        o = int(h["data_offset"])
        return self.data[o:o + n].reshape(int(h["active_channels"]), int(h["number_of_samples"]))

    @staticmethod
    def build(acqs, encoded, recon, ky_center, kz_center=0) -> "AcquisitionSet":
        """``acqs``: list of (dict of header fields, [nc, ns] complex array)."""
        hdr = np.zeros(len(acqs), HEADER_DTYPE)
        off = 0
        chunks = []
        for i, (h, d) in enumerate(acqs):
            d = np.ascontiguousarray(d, dtype=np.complex64)
            for k, v in h.items():
                hdr[i][k] = v
            hdr[i]["active_channels"], hdr[i]["number_of_samples"] = d.shape
            hdr[i]["data_offset"] = off
            off += d.size
            chunks.append(d.ravel())
        data = np.concatenate(chunks) if chunks else np.zeros(0, np.complex64)
        return AcquisitionSet(hdr, data, tuple(encoded), tuple(recon), ky_center, kz_center)


def oversampled_acquisitions(vol) -> AcquisitionSet:
    """An AcquisitionSet of a synth.OversampledVolume: one noise scan, then the
    sampled ky lines of every slice (2-D multi-slice: ``slice`` = z)."""
    nz, nl, nc, ex = vol.lines.shape
    acqs = [({"flags": ACQ_IS_NOISE_MEASUREMENT}, vol.noise)]
    for z in range(nz):
        for i in range(nl):
            acqs.append(({"kspace_encode_step_1": int(vol.ky_index[z, i]), "slice": z,
                          "center_sample": ex // 2}, vol.lines[z, i]))
    return AcquisitionSet.build(acqs, (ex, vol.ny, 1), (vol.rec_x, vol.ny, 1), vol.ny // 2)


def cartesian3d_acquisitions(kspace: np.ndarray, mask_rows: np.ndarray) -> AcquisitionSet:
    """An AcquisitionSet of 3-D Cartesian k-space [nc, nz, ny, nx]: every
    sampled ky line of every kz partition (``kspace_encode_step_2`` = kz), no
    noise scan, no readout oversampling."""
    nc, nz, ny, nx = kspace.shape
    rows = np.flatnonzero(mask_rows)
    acqs = []
    for z in range(nz):
        for r in rows:
            acqs.append(({"kspace_encode_step_1": int(r), "kspace_encode_step_2": z, "center_sample": nx // 2},
                         kspace[:, z, r, :]))
    return AcquisitionSet.build(acqs, (nx, ny, nz), (nx, ny, nz), ny // 2, nz // 2)


@dataclasses.dataclass
class ImageVolume:
    """strategy.rs:26-34."""
    data: np.ndarray
    strategy: str
    gfactor: np.ndarray | None = None


@dataclasses.dataclass
class CsRss:
    """strategy.rs:753-775: same public fields and defaults."""
    remove_oversampling: bool = True
    prewhiten: bool = True
    phase_correct: bool = True
    iters: int = 60
    lambda_: float = 0.01
    fft_mode: str = "auto"          # "auto" | "2d" | "3d"  (strategy.rs:72-79)
    crop_to_recon_matrix: bool = True

    def name(self) -> str:
        return "cs"

    def _cfg(self) -> _Cfg:
        return _Cfg(int(self.remove_oversampling), int(self.prewhiten), int(self.phase_correct), int(self.iters),
                    float(self.lambda_), {"auto": 0, "2d": 1, "3d": 2}[self.fft_mode],
                    int(self.crop_to_recon_matrix))

    def output_shape(self, ctx, acqs: AcquisitionSet) -> tuple:
        hdr = np.ascontiguousarray(acqs.headers, dtype=HEADER_DTYPE)
        s = _AcqSet(len(hdr), hdr.ctypes.data, acqs.data.ctypes.data if acqs.data.size else 1, acqs.data.size, 0,
                    *acqs.encoded, *acqs.recon, acqs.ky_center, acqs.kz_center)
        cfg = self._cfg()
        dims = (ctypes.c_int * 3)()
        ctx.check(ctx.lib.okscuda_csrss_reconstruct(ctx.handle, ctypes.byref(cfg), ctypes.byref(s), None, 0, dims))
        return tuple(dims)

    def reconstruct(self, ctx, acqs: AcquisitionSet, device_data=None, out=None) -> ImageVolume:
        """strategy.rs:782-891 through okscuda_csrss_reconstruct.  With
        ``device_data`` (a DeviceArray holding ``acqs.data``) the samples are
        read from device memory and the volume is written to ``out`` (a
        DeviceArray of ``output_shape``) without waiting for the GPU."""
        hdr = np.ascontiguousarray(acqs.headers, dtype=HEADER_DTYPE)
        data = acqs.data if acqs.data.flags["C_CONTIGUOUS"] else np.ascontiguousarray(acqs.data)
        s = _AcqSet(len(hdr), hdr.ctypes.data, device_data.ptr if device_data is not None else data.ctypes.data,
                    data.size, int(device_data is not None), *acqs.encoded, *acqs.recon, acqs.ky_center,
                    acqs.kz_center)
        cfg = self._cfg()
        dims = (ctypes.c_int * 3)()
        L = ctx.lib
        if device_data is not None:
            if out is None:
                out = ctx.empty(self.output_shape(ctx, acqs), np.float32)
            rc = L.okscuda_csrss_reconstruct(ctx.handle, ctypes.byref(cfg), ctypes.byref(s), out.ptr, out.size, dims)
            if rc != 0:
                raise OksError(rc, ctx.last_error())
            return ImageVolume(out, self.name())
        ctx.check(L.okscuda_csrss_reconstruct(ctx.handle, ctypes.byref(cfg), ctypes.byref(s), None, 0, dims))
        host = out if out is not None else np.empty(tuple(dims), np.float32)
        rc = L.okscuda_csrss_reconstruct(ctx.handle, ctypes.byref(cfg), ctypes.byref(s), host.ctypes.data,
                                         host.size, dims)
        if rc != 0:
            raise OksError(rc, ctx.last_error())
        return ImageVolume(host, self.name())
