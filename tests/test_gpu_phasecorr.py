"""Navigator phase correction (phasecorr.rs:61-169) inside the CsRss pipeline
(strategy.rs:782-815: prewhitening, then the navigator phasor, then
oversampling removal) through the C-ABI, against the FP64 pipeline oracle.

TSE-like data: the lines of each (slice, segment) carry a linear phase error
phi(k); per bin, navigator scans sample exp(i phi(k)) times positive channel
weights, so their coil sum has phase phi exactly and the correction removes
the error.  Tolerance: NRMSE <= 1e-4 on the magnitude volume.
"""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import strategy_ref
from openkspace_b200 import synth
from openkspace_b200.strategy import (ACQ_IS_NOISE_MEASUREMENT, ACQ_IS_PHASECORR_DATA, AcquisitionSet, CsRss)

pytestmark = pytest.mark.gpu
TOL = 1e-4
ETL = 4          # echoes per train: segment = line index % ETL
ITERS, LAM = 12, 0.005


def tse_acquisitions(vol, corrupt=True, navigators=True, nav_slice=None, nav_ns=None, extra=True, seed=5):
    """AcquisitionSet of a synth.OversampledVolume with per-(slice, segment)
    phase errors on the image lines and navigator scans measuring them.
    nav_slice: tag every navigator with this slice (65535: the fallback bin).
    nav_ns: navigator length (shorter than the lines: only their start is corrected)."""
    rng = np.random.default_rng(seed)
    nz, nl, nc, ex = vol.lines.shape
    k = np.arange(ex)
    phase = {}
    for z in range(nz):
        for s in range(ETL):
            zz = z if nav_slice is None else 0
            if (zz, s) not in phase:
                a, b = rng.uniform(-np.pi, np.pi), rng.uniform(-2.0, 2.0)
                phase[(zz, s)] = a + b * np.pi * (k - ex / 2) / ex
    acqs = [({"flags": ACQ_IS_NOISE_MEASUREMENT}, vol.noise)]
    if navigators:
        ns = ex if nav_ns is None else nav_ns
        for z in range(nz if nav_slice is None else 1):
            for s in range(ETL):
                phi = phase[(z, s)][:ns]
                for rep in range(2):
                    w = rng.uniform(0.5, 2.0, nc)[:, None]
                    g = 1.0 + 0.5 * np.cos(2 * np.pi * (rep + 1) * np.arange(ns) / ns)
                    nav = (w * g * np.exp(1j * phi)).astype(np.complex64)
                    acqs.append(({"flags": ACQ_IS_PHASECORR_DATA, "slice": z if nav_slice is None else nav_slice,
                                  "segment": s}, nav))
                if extra and z == 0 and s == 0:
                    # another length in a bin that exists: dropped (phasecorr.rs:92-98)
                    acqs.append(({"flags": ACQ_IS_PHASECORR_DATA, "slice": 0 if nav_slice is None else nav_slice,
                                  "segment": 0}, rng.standard_normal((nc, ns // 2)).astype(np.complex64)))
    for z in range(nz):
        for i in range(nl):
            s = i % ETL
            line = vol.lines[z, i]
            if corrupt:
                line = (line * np.exp(1j * phase[(z if nav_slice is None else 0, s)])[None]).astype(np.complex64)
            acqs.append(({"kspace_encode_step_1": int(vol.ky_index[z, i]), "slice": z, "segment": s,
                          "center_sample": ex // 2}, line))
    return AcquisitionSet.build(acqs, (ex, vol.ny, 1), (vol.rec_x, vol.ny, 1), vol.ny // 2)


def oracle(a, phase_correct=True):
    return strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                          iters=ITERS, lam=LAM, phase_correct=phase_correct)


@pytest.fixture(scope="module")
def vol():
    return synth.oversampled_volume(nz=2, nc=4, ny=64, enc_x=128, rec_x=64)


@pytest.mark.parametrize("case", ["per_slice", "fallback_bin", "short_navigators"])
def test_phase_correction_matches_oracle(ctx, vol, case):
    kw = {"per_slice": {}, "fallback_bin": {"nav_slice": 65535}, "short_navigators": {"nav_ns": 80}}[case]
    a = tse_acquisitions(vol, **kw)
    got = CsRss(iters=ITERS, lambda_=LAM).reconstruct(ctx, a).data
    want = oracle(a)
    assert got.shape == want.shape == (2, 64, 64)
    assert o64.nrmse(got, want) <= TOL


def test_phase_correction_restores_the_clean_reconstruction(ctx, vol):
    """With full-length navigators the corrected lines are the clean ones (the
    phasor commutes with the channel-mixing prewhitener)."""
    s = CsRss(iters=ITERS, lambda_=LAM)
    fixed = s.reconstruct(ctx, tse_acquisitions(vol)).data
    clean = s.reconstruct(ctx, tse_acquisitions(vol, corrupt=False, navigators=False)).data
    corrupted = CsRss(iters=ITERS, lambda_=LAM, phase_correct=False).reconstruct(ctx, tse_acquisitions(vol)).data
    assert o64.nrmse(fixed, clean) <= TOL
    assert o64.nrmse(corrupted, clean) > 1e-2


def test_phase_correct_off_ignores_navigators(ctx, vol):
    a = tse_acquisitions(vol)
    got = CsRss(iters=ITERS, lambda_=LAM, phase_correct=False).reconstruct(ctx, a).data
    assert o64.nrmse(got, oracle(a, phase_correct=False)) <= TOL


def test_phase_correction_with_device_resident_samples(ctx, vol):
    """data_on_device: the navigators are gathered device to device; same
    volume as the host-sample call."""
    a = tse_acquisitions(vol)
    s = CsRss(iters=ITERS, lambda_=LAM)
    host = s.reconstruct(ctx, a).data
    d = ctx.to_device(a.data)
    dev = s.reconstruct(ctx, a, device_data=d).data.to_host()
    assert np.array_equal(dev, host)


def test_navigators_with_fewer_channels_than_the_lines(ctx, vol):
    """The coil sum runs over the navigator's own channels (phasecorr.rs:79-86);
    the phasor multiplies every channel of the image line (:161-168)."""
    a = tse_acquisitions(vol)
    h = a.headers.copy()
    data = a.data.copy()
    nav = np.flatnonzero(h["flags"] & ACQ_IS_PHASECORR_DATA)
    # keep the first two channels of every navigator in place (same offsets)
    for i in nav:
        h[i]["active_channels"] = 2
    b = AcquisitionSet(h, data, a.encoded, a.recon, a.ky_center, a.kz_center)
    got = CsRss(iters=ITERS, lambda_=LAM).reconstruct(ctx, b).data
    assert o64.nrmse(got, oracle(b)) <= TOL
