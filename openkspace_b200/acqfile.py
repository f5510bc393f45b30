"""Acquisition stream files: the rows of an ISMRMRD dataset without HDF5.

``write_acquisitions`` serialises an ``AcquisitionSet`` (XML header with the
encoding block, then per acquisition the packed 340-byte AcquisitionHeader,
trajectory and samples -- the layout documented at okscuda_raw_open in
include/okscuda.h).  ``read_acquisitions`` opens such a file through the
C-ABI reader (okscuda_raw_open: headers, then the samples straight into one
pinned host buffer) and returns an ``AcquisitionSet`` over that memory, ready
for ``CsRss.reconstruct``.
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

from . import _lib
from ._lib import OksError
from .strategy import HEADER_DTYPE, AcquisitionSet, _AcqSet

MAGIC = b"OKSACQ1\x00"
HEADER_BYTES = 340


def ismrmrd_xml(encoded, recon, ky_center: int, kz_center: int = 0, receiver_channels: int = 0) -> str:
    """The encoding block of an ISMRMRD XML header (the fields header.rs reads)."""
    ex, ey, ez = encoded
    rx, ry, rz = recon
    return ('<?xml version="1.0"?>\n<ismrmrdHeader xmlns="http://www.ismrm.org/ISMRMRD">\n'
            f"  <acquisitionSystemInformation><receiverChannels>{receiver_channels}</receiverChannels>"
            "</acquisitionSystemInformation>\n"
            "  <encoding>\n"
            f"    <encodedSpace><matrixSize><x>{ex}</x><y>{ey}</y><z>{ez}</z></matrixSize></encodedSpace>\n"
            f"    <reconSpace><matrixSize><x>{rx}</x><y>{ry}</y><z>{rz}</z></matrixSize></reconSpace>\n"
            "    <encodingLimits>\n"
            f"      <kspace_encoding_step_1><minimum>0</minimum><maximum>{max(ey - 1, 0)}</maximum>"
            f"<center>{ky_center}</center></kspace_encoding_step_1>\n"
            f"      <kspace_encoding_step_2><minimum>0</minimum><maximum>{max(ez - 1, 0)}</maximum>"
            f"<center>{kz_center}</center></kspace_encoding_step_2>\n"
            "    </encodingLimits>\n"
            "    <trajectory>cartesian</trajectory>\n"
            "  </encoding>\n</ismrmrdHeader>\n")


def pack_header(h) -> bytes:
    """One packed little-endian AcquisitionHeader (acquisition.rs:33-59 field
    order); fields the cs path does not read are zero."""
    b = bytearray(HEADER_BYTES)
    struct.pack_into("<H", b, 0, 1)                                   # version
    struct.pack_into("<Q", b, 2, int(h["flags"]))
    struct.pack_into("<HHH", b, 34, int(h["number_of_samples"]), int(h["active_channels"]),
                     int(h["active_channels"]))                       # number_of_samples, available, active
    struct.pack_into("<HHHHH", b, 168, int(h["discard_pre"]), int(h["discard_post"]), int(h["center_sample"]),
                     0, 0)                                            # ..., encoding_space_ref, trajectory_dimensions
    struct.pack_into("<HH", b, 242, int(h["kspace_encode_step_1"]), int(h["kspace_encode_step_2"]))
    struct.pack_into("<H", b, 248, int(h["slice"]))
    struct.pack_into("<H", b, 258, int(h["segment"]))
    return bytes(b)


def write_acquisitions(path: str, acqs: AcquisitionSet, receiver_channels: int = 0):
    xml = ismrmrd_xml(acqs.encoded, acqs.recon, acqs.ky_center, acqs.kz_center, receiver_channels).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(xml)))
        f.write(xml)
        f.write(struct.pack("<Q", len(acqs.headers)))
        for i in range(len(acqs.headers)):
            h = acqs.headers[i]
            f.write(pack_header(h))
            f.write(np.ascontiguousarray(acqs.acquisition(i), dtype="<c8").tobytes())


class AcquisitionFile:
    """An open acquisition stream file (okscuda_raw_*): ``acqs`` is an
    AcquisitionSet whose headers and samples are views of the reader's
    memory (pinned when a device is present), valid until ``close``."""

    def __init__(self, path: str):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.okscuda_raw_open(os.fsencode(path), ctypes.byref(h))
        if rc != 0:
            raise OksError(rc, f"reading acquisitions from {path}")
        self.handle = h.value
        s = _AcqSet()
        self.lib.okscuda_raw_acq_set(self.handle, ctypes.byref(s))
        n = int(s.n_acq)
        hdr = (np.ctypeslib.as_array((ctypes.c_uint8 * (n * HEADER_DTYPE.itemsize)).from_address(s.headers))
               .view(HEADER_DTYPE) if n else np.zeros(0, HEADER_DTYPE))
        data = (np.ctypeslib.as_array((ctypes.c_float * (2 * s.data_len)).from_address(s.data)).view(np.complex64)
                if s.data_len else np.zeros(0, np.complex64))
        self.acqs = AcquisitionSet(hdr, data, (s.enc_x, s.enc_y, s.enc_z), (s.rec_x, s.rec_y, s.rec_z),
                                   s.ky_center, s.kz_center)
        rc_ch, xl = ctypes.c_int(), ctypes.c_int()
        self.lib.okscuda_raw_info(self.handle, ctypes.byref(rc_ch), ctypes.byref(xl))
        self.receiver_channels = rc_ch.value

    def close(self):
        if self.handle:
            self.lib.okscuda_raw_close(self.handle)
            self.handle = None
            self.acqs = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_acquisitions(path: str) -> AcquisitionFile:
    return AcquisitionFile(path)
