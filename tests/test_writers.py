"""Output writers on the host (no GPU): the NIfTI-1 file of
main.rs:1033-1074 (the reference's own test nifti_round_trip_header,
main.rs:1160-1200, restated), the PNG encoder (decoded back with zlib), and
the oracle's percentile() pinned to hand-computed cases of main.rs:1147-1153."""
import struct
import zlib

import numpy as np

from openkspace_b200 import writers
from oracle import writers_ref


def test_nifti_round_trip_header(tmp_path):
    vol = np.full((4, 8, 16), 1.0, np.float32)
    path = tmp_path / "test.nii"
    writers.write_nifti_volume(vol, str(path))
    raw = path.read_bytes()
    h = writers_ref.nifti_header(raw)
    assert h["sizeof_hdr"] == 348
    assert h["dim"][:4] == (3, 16, 8, 4)               # nx, ny, nz (x fastest)
    assert h["dim"][4:] == (1, 1, 1, 1)
    assert h["datatype"] == 16 and h["bitpix"] == 32
    assert h["pixdim"][:4] == (1.0, 1.0, 1.0, 1.0)
    assert abs(h["vox_offset"] - 352.0) < 1e-6
    assert h["scl_slope"] == 1.0
    assert h["magic"] == b"n+1\x00"
    assert len(raw) == 352 + 4 * 8 * 16 * 4
    assert raw[348:352] == b"\x00" * 4


def test_nifti_data_order(tmp_path):
    vol = np.arange(2 * 3 * 5, dtype=np.float32).reshape(2, 3, 5)
    path = tmp_path / "v.nii"
    writers.write_nifti_volume(vol, str(path))
    data = np.frombuffer(path.read_bytes()[352:], dtype="<f4")
    assert np.array_equal(data, vol.ravel())            # C order of [nz, ny, nx] = x fastest


def _decode_png(raw: bytes):
    assert raw[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(raw):
        n = struct.unpack_from(">I", raw, pos)[0]
        typ = raw[pos + 4:pos + 8]
        data = raw[pos + 8:pos + 8 + n]
        assert struct.unpack_from(">I", raw, pos + 8 + n)[0] == zlib.crc32(typ + data)
        chunks.setdefault(typ, b"")
        chunks[typ] += data
        pos += 12 + n
    w, h, depth, ctype = struct.unpack(">IIBB", chunks[b"IHDR"][:10])
    rows = zlib.decompress(chunks[b"IDAT"])
    img = np.frombuffer(rows, np.uint8).reshape(h, w + 1)
    assert np.all(img[:, 0] == 0)
    return depth, ctype, img[:, 1:]


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    for h, w in ((1, 1), (3, 7), (300, 320), (257, 300)):     # > 65535 raw bytes: several stored blocks
        g = rng.integers(0, 256, (h, w), dtype=np.uint8)
        path = tmp_path / f"g{h}x{w}.png"
        writers.write_png(g, str(path))
        depth, ctype, back = _decode_png(path.read_bytes())
        assert depth == 8 and ctype == 0
        assert np.array_equal(back, g)


def test_oracle_percentile_pins():
    v = np.array([5.0, 1.0, 3.0, 2.0, 4.0], np.float32)
    assert writers_ref.percentile(v, 0.0) == 1.0
    assert writers_ref.percentile(v, 100.0) == 5.0
    assert writers_ref.percentile(v, 50.0) == 3.0
    assert writers_ref.percentile(v, 12.5) == 2.0          # 0.125 * 4 = 0.5 rounds away from zero
    assert writers_ref.percentile(v, 12.4) == 1.0
    assert writers_ref.percentile([], 50.0) == 0.0
    assert writers_ref.percentile([7.0], 99.0) == 7.0


def test_oracle_window_pins():
    img = np.array([-1.0, 0.0, 0.5, 1.0, 2.0, np.nan], np.float32)
    assert list(writers_ref.window_u8(img, 0.0, 1.0, False)) == [0, 0, 128, 255, 255, 0]
    g = writers_ref.window_u8(img, 0.0, 1.0, True)
    assert g[2] == int(np.floor(np.float32(0.5) ** np.float32(0.9) * 255 + 0.5))
    assert list(writers_ref.window_u8(np.array([3.0], np.float32), 3.0, 3.0, False)) == [0]   # hi = lo + eps
