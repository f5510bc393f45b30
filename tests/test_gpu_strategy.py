"""Feeding stages (prewhitening fit/apply, oversampling removal, kz IFFT,
odd-size IFFT) and the drop-in CsRss strategy, against the oracle, through
the C-ABI.  Tolerances: 1e-5 relative for single transforms and the FP64
whitening matrix, NRMSE <= 1e-4 for reconstructions."""
import ctypes

import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import csref
from oracle import strategy_ref
from openkspace_b200 import OksError, _lib, synth
from openkspace_b200.strategy import (ACQ_IS_NOISE_MEASUREMENT, ACQ_IS_REVERSE, AcquisitionSet, CsRss,
                                      oversampled_acquisitions)
from tests.conftest import crandn, rel_l2
from tests.test_oracle_pins import lcg_whitening_fixture

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


def fit(ctx, noise, total=0):
    nc, ns = noise.shape
    d = ctx.to_device(noise)
    w = ctx.empty((nc, nc))
    rc = ctx.lib.okscuda_prewhiten_fit(ctx.handle, d.ptr, nc, ns, total, w.ptr)
    return rc, (w.to_host() if rc == 0 else None)


def test_prewhiten_fit_lcg_fixture(ctx):
    """prewhiten.rs:218-302 on the device: FP64 W, whitened covariance ~ I."""
    data = lcg_whitening_fixture()
    rc, w = fit(ctx, data)
    assert rc == 0
    assert rel_l2(w, o64.prewhitener_from_noise([data])) < 1e-6
    assert rel_l2(w, csref.prewhiten_fit(data)) < 1e-4
    d = ctx.to_device(data[None])
    dw = ctx.to_device(w)   # keep the device array alive until the call has been made
    ctx.check(ctx.lib.okscuda_prewhiten_apply(ctx.handle, dw.ptr, d.ptr, 1, 4, data.shape[1]))
    out = d.to_host()[0]
    cov = out @ np.conj(out.T) / (data.shape[1] - 1)
    assert np.max(np.abs(cov - np.eye(4))) < 0.08


@pytest.mark.parametrize("nc", [1, 8, 15, 32, 64])
def test_prewhiten_fit_apply_sizes(ctx, rng, nc):
    psi = synth.noise_covariance(nc, 50.0, rng)
    ev, evec = np.linalg.eigh(psi)
    sq = (evec * np.sqrt(ev)) @ np.conj(evec.T)
    noise = (sq @ crandn(rng, (nc, 300))).astype(np.complex64)
    rc, w = fit(ctx, noise)
    assert rc == 0
    assert rel_l2(w, o64.prewhitener_from_noise([noise])) < 1e-5
    data = crandn(rng, (5, nc, 96))
    d = ctx.to_device(data)
    dw = ctx.to_device(w)
    ctx.check(ctx.lib.okscuda_prewhiten_apply(ctx.handle, dw.ptr, d.ptr, 5, nc, 96))
    assert rel_l2(d.to_host(), o64.prewhiten_apply(w.astype(np.complex128), data)) < 1e-5


def test_prewhiten_skip_cases(ctx, rng):
    rc, _ = fit(ctx, crandn(rng, (4, 3)))                 # too few samples
    assert rc == _lib.OKS_ESKIP
    rc, _ = fit(ctx, np.ones((3, 10), np.complex64))      # singular covariance
    assert rc == _lib.OKS_ENOTPD
    # samples of scans with another channel count still count towards the
    # total (prewhiten.rs:58): the size check passes, the rank-3 covariance
    # of 4 channels then fails Cholesky
    rc, _ = fit(ctx, crandn(rng, (4, 3)), total=40)
    assert rc == _lib.OKS_ENOTPD
    rc, w = fit(ctx, crandn(rng, (4, 6)), total=40)
    assert rc == 0
    data = crandn(rng, (4, 6))
    rc, w = fit(ctx, data, total=40)
    want = o64.cholesky_lower(data.astype(np.complex128) @ np.conj(data.T).astype(np.complex128) / 39.0)
    assert rel_l2(w, o64.invert_lower_triangular(want)) < 1e-5


@pytest.mark.parametrize("enc,rec", [(16, 8), (640, 320), (384, 128), (30, 10), (7, 1)])
def test_os_remove(ctx, rng, enc, rec):
    d = crandn(rng, (3, 4, enc))
    out = ctx.empty((3, 4, rec))
    dd = ctx.to_device(d)
    ctx.check(ctx.lib.okscuda_os_remove(ctx.handle, dd.ptr, out.ptr, 12, enc, rec))
    assert rel_l2(out.to_host(), o64.oversampling_apply(d, enc, rec)) < 1e-5


def test_os_remove_dc_and_invalid(ctx):
    d = np.zeros((1, 16), np.complex64)
    d[0, 8] = 10.0
    out = ctx.empty((1, 8))
    dd = ctx.to_device(d)
    ctx.check(ctx.lib.okscuda_os_remove(ctx.handle, dd.ptr, out.ptr, 1, 16, 8))
    o = out.to_host()[0]
    assert abs(o[4] - 5.0) < 1e-4 and np.max(np.abs(np.delete(o, 4))) < 1e-4
    assert ctx.lib.okscuda_os_remove(ctx.handle, dd.ptr, out.ptr, 1, 300, 256) == _lib.OKS_ESKIP


@pytest.mark.parametrize("nz", [4, 5, 192, 1])
def test_ifft1_kz(ctx, rng, nz):
    k = crandn(rng, (2, nz, 6, 10))
    d = ctx.to_device(k)
    ctx.check(ctx.lib.okscuda_ifft1_kz(ctx.handle, d.ptr, 2, nz, 6, 10))
    assert rel_l2(d.to_host(), o64.ifft1_inplace(k, 1)) < 1e-5


@pytest.mark.parametrize("ny,nx", [(5, 7), (8, 6), (1, 9)])
def test_ifft2(ctx, rng, ny, nx):
    k = crandn(rng, (3, ny, nx))
    d = ctx.to_device(k)
    ctx.check(ctx.lib.okscuda_ifft2(ctx.handle, d.ptr, 3, ny, nx))
    assert rel_l2(d.to_host(), o64.ifft2_inplace(k, (1, 2))) < 1e-5


# ------------------------------------------------------------------ CsRss
def small_acqset(rng, nc=4, ny=24, enc=32, rec=16, nz=3, reverse=False, discard=0, dup=False, three_d=False,
                 noise=True):
    acqs = []
    if noise:
        acqs.append(({"flags": ACQ_IS_NOISE_MEASUREMENT}, crandn(rng, (nc, 64)) * 0.1))
    for z in range(nz):
        rows = np.flatnonzero(rng.random(ny) < 0.5)
        rows = np.union1d(rows, np.arange(ny // 2 - 2, ny // 2 + 2))
        for r in rows:
            h = {"kspace_encode_step_1": int(r), "center_sample": enc // 2 + discard, "discard_pre": discard}
            if three_d:
                h["kspace_encode_step_2"] = z
            else:
                h["slice"] = z
            if reverse and r % 3 == 0:
                h["flags"] = ACQ_IS_REVERSE
            acqs.append((h, crandn(rng, (nc, enc + discard))))
            if dup and r % 4 == 0:
                acqs.append((h, crandn(rng, (nc, enc + discard))))   # later duplicate: dropped
    return AcquisitionSet.build(acqs, (enc, ny, nz if three_d else 1), (rec, ny - 4, nz if three_d else 1),
                                ny // 2, nz // 2 if three_d else 0)


def run_both(ctx, a: AcquisitionSet, **kw):
    s = CsRss(**kw)
    got = s.reconstruct(ctx, a).data
    want = strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                          iters=s.iters, lam=s.lambda_,
                                          remove_oversampling=s.remove_oversampling, prewhiten=s.prewhiten,
                                          fft_mode=s.fft_mode, crop=s.crop_to_recon_matrix)
    assert got.shape == want.shape
    return got, want


@pytest.mark.parametrize("kw", [dict(), dict(reverse=True), dict(discard=3), dict(dup=True),
                                dict(three_d=True), dict(noise=False), dict(enc=24, rec=24)])
def test_csrss_matches_oracle(ctx, rng, kw):
    a = small_acqset(rng, **kw)
    got, want = run_both(ctx, a, iters=15, lambda_=0.01)
    assert o64.nrmse(got, want) < TOL_CS


def test_csrss_options(ctx, rng):
    a = small_acqset(rng)
    for kw in [dict(remove_oversampling=False), dict(prewhiten=False), dict(crop_to_recon_matrix=False),
               dict(fft_mode="3d"), dict(iters=0)]:
        got, want = run_both(ctx, a, **{"iters": 8, "lambda_": 0.02, **kw})
        assert o64.nrmse(got, want) < TOL_CS, kw


def test_csrss_odd_dims_fallback(ctx, rng):
    a = small_acqset(rng, ny=23, enc=18, rec=9)
    got, want = run_both(ctx, a, iters=10)
    assert o64.nrmse(got, want) < 1e-5


def test_csrss_errors(ctx, rng):
    a = small_acqset(rng)
    with pytest.raises(OksError) as e:
        noise_only = AcquisitionSet(a.headers[:1].copy(), a.data, a.encoded, a.recon, a.ky_center)
        CsRss().reconstruct(ctx, noise_only)
    assert e.value.code == _lib.OKS_EINVAL
    assert CsRss().name() == "cs"
    assert ctx.lib.okscuda_csrss_name() == b"cs"


def test_csrss_oversampled_precision_volume_small(ctx):
    """The precision workload's pipeline at reduced size: 15 coils, 2x
    readout oversampling, correlated noise + 256 noise samples, R = 4 with an
    8 % centre, lambda 0.005.  Lines are placed at the central half of a
    2x-wide k-space row (reader.rs:265 sizes kx from the raw readout)."""
    vol = synth.oversampled_volume(nz=2, nc=15, ny=64, enc_x=96, rec_x=48, workload=1)
    a = oversampled_acquisitions(vol)
    got, want = run_both(ctx, a, iters=20, lambda_=0.005)
    assert got.shape == (2, 64, 48)
    assert o64.nrmse(got, want) < TOL_CS
