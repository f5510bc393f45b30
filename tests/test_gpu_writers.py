"""Output writers on the device against the oracle's restatement of
main.rs:1095-1153: the percentile is the exact element (radix select against
the sorted array, bit for bit) on ragged sizes, duplicates, negative values
and signed zeros; the 8-bit window is byte-exact in the linear form and
within one grey level in the gamma form (CUDA's powf and the host's may
differ in the last bit, which moves round(x * 255) by one at most); a
reconstructed slice goes to PNG and NIfTI end to end."""
import numpy as np
import pytest

from openkspace_b200 import synth, writers
from oracle import writers_ref
from tests.test_writers import _decode_png

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 7, 1000, 117760, 1 << 20])
def test_percentile_is_the_exact_element(ctx, n):
    rng = np.random.default_rng(n)
    v = (rng.standard_normal(n) * 10).astype(np.float32)
    if n > 10:
        v[: n // 10] = v[n // 5]                         # duplicates
        v[n // 3] = -0.0
        v[n // 3 + 1] = 0.0
    d = ctx.to_device(v)
    for pct in (0.0, 0.5, 1.0, 12.5, 50.0, 99.0, 99.5, 100.0):
        got = np.float32(writers.percentile(ctx, d, pct))
        want = writers_ref.percentile(v, pct)
        assert got == want or (got == 0 and want == 0), (n, pct, got, want)


def test_percentile_of_magnitudes_and_empty(ctx):
    rng = np.random.default_rng(4)
    v = np.abs(rng.standard_normal((368, 320))).astype(np.float32)
    for pct in (1.0, 99.5):
        assert np.float32(writers.percentile(ctx, v, pct)) == writers_ref.percentile(v, pct)
    assert writers.percentile(ctx, np.zeros(0, np.float32), 50.0) == 0.0


def test_window_linear_exact_and_gamma_within_one(ctx):
    rng = np.random.default_rng(6)
    img = (rng.random((300, 257)) * 3 - 0.5).astype(np.float32)
    img[0, :5] = [np.nan, np.inf, -np.inf, 0.0, 2.0]
    lin = writers.window_u8(ctx, img, 0.0, 2.0, False)
    assert np.array_equal(lin, writers_ref.window_u8(img, 0.0, 2.0, False))
    gam = writers.window_u8(ctx, img, 0.1, 1.7, True)
    want = writers_ref.window_u8(img, 0.1, 1.7, True)
    diff = np.abs(gam.astype(int) - want.astype(int))
    assert diff.max() <= 1
    assert np.mean(diff) < 1e-3


def test_reconstructed_slice_to_png_and_nifti(ctx, tmp_path):
    s = synth.make_slice(128, 128, 4, 4.0, 12, seed=7)
    rss = ctx.cs_slice(s.kspace, s.mask2d, 20, 0.01)
    d = ctx.to_device(rss)
    g = writers.write_png_windowed(ctx, d, str(tmp_path / "slice_0000.png"), 1.0, 99.5)
    _, _, back = _decode_png((tmp_path / "slice_0000.png").read_bytes())
    assert np.array_equal(back, g)
    want = writers_ref.png_windowed(rss, 1.0, 99.5)
    assert np.abs(g.astype(int) - want.astype(int)).max() <= 1
    writers.write_nifti_volume(d.to_host()[None], str(tmp_path / "v.nii"))
    data = np.frombuffer((tmp_path / "v.nii").read_bytes()[352:], dtype="<f4")
    assert np.array_equal(data, rss.ravel())
