"""Acquisition stream files (okscuda_raw_open, no HDF5): a written set reads
back field for field and sample for sample; the XML header's encoding block
is parsed with the reference's tag-path rules -- the reference's own header
test (header.rs:210-264, restated) on its sample XML; malformed files are
refused.  Host only: runs without a GPU."""
import struct

import numpy as np
import pytest

from openkspace_b200 import OksError, _lib
from openkspace_b200.acqfile import MAGIC, read_acquisitions, write_acquisitions
from openkspace_b200.strategy import ACQ_IS_NOISE_MEASUREMENT, ACQ_IS_REVERSE, AcquisitionSet

_lib.load()

SAMPLE_XML = """<?xml version="1.0"?>
    <ismrmrdHeader xmlns="http://www.ismrm.org/ISMRMRD">
      <acquisitionSystemInformation>
        <systemVendor>GE MEDICAL SYSTEMS</systemVendor>
        <systemModel>Orchestra SDK</systemModel>
        <systemFieldStrength_T>3.000000</systemFieldStrength_T>
        <receiverChannels>8</receiverChannels>
      </acquisitionSystemInformation>
      <encoding>
        <encodedSpace>
          <matrixSize><x>352</x><y>216</y><z>30</z></matrixSize>
          <fieldOfView_mm><x>280</x><y>280</y><z>4.5</z></fieldOfView_mm>
        </encodedSpace>
        <reconSpace>
          <matrixSize><x>512</x><y>512</y><z>0</z></matrixSize>
          <fieldOfView_mm><x>280</x><y>280</y><z>4.5</z></fieldOfView_mm>
        </reconSpace>
        <encodingLimits>
          <kspace_encoding_step_1><minimum>0</minimum><maximum>215</maximum><center>108</center></kspace_encoding_step_1>
          <kspace_encoding_step_2><minimum>0</minimum><maximum>0</maximum><center>0</center></kspace_encoding_step_2>
          <slice><minimum>0</minimum><maximum>29</maximum><center>15</center></slice>
        </encodingLimits>
        <trajectory>cartesian</trajectory>
      </encoding>
    </ismrmrdHeader>"""


def _small_set():
    rng = np.random.default_rng(3)
    acqs = [({"flags": ACQ_IS_NOISE_MEASUREMENT}, (rng.standard_normal((4, 32)) + 1j).astype(np.complex64))]
    for z in range(2):
        for ky in (1, 5, 8, 11):
            d = (rng.standard_normal((4, 24)) + 1j * rng.standard_normal((4, 24))).astype(np.complex64)
            acqs.append(({"kspace_encode_step_1": ky, "slice": z, "center_sample": 12, "segment": ky % 2,
                          "discard_pre": 1, "discard_post": 2, "flags": ACQ_IS_REVERSE if ky == 5 else 0}, d))
    return AcquisitionSet.build(acqs, (24, 16, 1), (20, 16, 1), 8)


def test_round_trip(tmp_path):
    a = _small_set()
    p = str(tmp_path / "a.oksacq")
    write_acquisitions(p, a, receiver_channels=4)
    with read_acquisitions(p) as f:
        b = f.acqs
        assert b.encoded == a.encoded and b.recon == a.recon
        assert b.ky_center == 8 and b.kz_center == 0
        assert f.receiver_channels == 4
        assert len(b.headers) == len(a.headers)
        for name in a.headers.dtype.names:
            assert np.array_equal(b.headers[name], a.headers[name]), name
        assert np.array_equal(b.data, a.data)


def test_reference_header_sample(tmp_path):
    p = tmp_path / "h.oksacq"
    x = SAMPLE_XML.encode()
    p.write_bytes(MAGIC + struct.pack("<I", len(x)) + x + struct.pack("<Q", 0))
    with read_acquisitions(str(p)) as f:
        assert f.receiver_channels == 8
        assert f.acqs.encoded == (352, 216, 30)
        assert f.acqs.recon == (512, 512, 0)
        assert f.acqs.ky_center == 108 and f.acqs.kz_center == 0
        assert len(f.acqs.headers) == 0


def test_malformed_files_are_refused(tmp_path):
    a = _small_set()
    p = tmp_path / "a.oksacq"
    write_acquisitions(str(p), a)
    raw = p.read_bytes()
    for bad in (b"NOTMAGIC" + raw[8:], raw[:-10], raw[:20]):
        q = tmp_path / "bad.oksacq"
        q.write_bytes(bad)
        with pytest.raises(OksError) as e:
            read_acquisitions(str(q))
        assert e.value.code == _lib.OKS_EINVAL
    with pytest.raises(OksError):
        read_acquisitions(str(tmp_path / "missing.oksacq"))
