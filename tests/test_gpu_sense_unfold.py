"""SENSE unfolding and g-factor on the device (okscuda_sense_unfold,
sense.rs:64-252): bit-identical to the FP32 C restatement that follows the
reference's operation order (the kernel uses explicitly rounded f32
operations, no fused multiply-adds), within 1e-5 relative L2 of the FP64
oracle, and the reference's own tests (R = 2 phantom NRMSE < 0.1, R = 1
pass-through, unit g-factor) through the device."""
import numpy as np
import pytest

from oracle import csref
from oracle import sense_fp64 as sref
from openkspace_b200 import OksError, _lib, synth
from tests.test_oracle_pins import _sense_r2_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nc,ny,nx,r,ridge", [(4, 32, 24, 2, 1e-5), (8, 96, 70, 3, 1e-3), (12, 128, 96, 4, 1e-4),
                                               (6, 60, 33, 6, 1e-3), (16, 64, 40, 8, 1e-3), (3, 9, 5, 1, 0.0),
                                               (20, 60, 33, 6, 1e-3)])
def test_unfold_matches_fp32_port_bitwise_and_fp64(ctx, nc, ny, nx, r, ridge):
    rng = np.random.default_rng(ny + r)
    maps = (rng.standard_normal((nc, ny, nx)) + 1j * rng.standard_normal((nc, ny, nx))).astype(np.complex64)
    al = (rng.standard_normal((nc, ny, nx)) + 1j * rng.standard_normal((nc, ny, nx))).astype(np.complex64)
    maps[:, :2, :3] = 0                                  # background: singular systems stay zero
    got, g = ctx.sense_unfold(al, maps, r, ridge, gfactor=True)
    want, gw = csref.sense_unfold(al, maps, r, ridge, gfactor=True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(g.view(np.uint32), gw.view(np.uint32))
    w64, g64 = sref.sense_unfold_1d(al, maps, r, ridge, gfactor=True)
    # f32 solves of r x r systems: random maps with as few coils as R (nc = 6,
    # R = 6) make them ill-conditioned, so the FP64 bound is 1e-4 there
    tol = 1e-5 if nc >= 2 * r else 1e-4
    assert np.linalg.norm(got - w64) / np.linalg.norm(w64) < tol
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < tol


def test_reference_cases_on_the_device(ctx):
    truth, maps, aliased, r = _sense_r2_case()
    out, _ = ctx.sense_unfold(aliased, maps, r, 1e-5)
    m = np.abs(out)
    assert np.sqrt(np.sum((truth - m) ** 2) / np.sum(truth ** 2)) < 0.1
    maps1 = np.ones((2, 8, 6), np.complex64)
    y, x = np.meshgrid(np.arange(8), np.arange(6), indexing="ij")
    al1 = np.stack([np.sin(y * 0.1 + x * 0.05 + c) for c in range(2)]).astype(np.complex64)
    out1, g1 = ctx.sense_unfold(al1, maps1, 1, 0.0, gfactor=True)
    assert np.abs(out1 - al1.mean(0)).max() < 1e-4
    assert np.abs(g1 - 1.0).max() < 1e-5


def test_walsh_maps_then_unfold(ctx):
    """The sense strategy's chain on a synthetic slice: Walsh maps of the
    device SENSE path, aliased images of a regular R = 2 mask, unfold."""
    s = synth.make_slice(128, 48, 6, 4.0, 12, seed=3)
    _, _, maps, _ = ctx.sense_cs(s.kspace, s.mask2d, 1, 0.0)
    k = np.array(s.kspace)
    m = np.zeros(128, bool)
    m[::2] = True
    k[:, ~m, :] = 0
    al = np.fft.ifft(k, axis=1).astype(np.complex64)
    got, _ = ctx.sense_unfold(al, maps, 2, 1e-4)
    want, _ = csref.sense_unfold(al, maps, 2, 1e-4)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_errors(ctx):
    z = np.zeros((2, 10, 4), np.complex64)
    for r, code in ((0, _lib.OKS_EINVAL), (3, _lib.OKS_ESHAPE), (10, _lib.OKS_ENOTSUP)):
        with pytest.raises(OksError) as e:
            ctx.sense_unfold(z, z, r, 0.0)
        assert e.value.code == code
