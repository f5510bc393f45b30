"""The precision workload at its full per-slice size -- 15 coils, 640 x 368
readout-oversampled k-space, R = 4 with an 8 % centre, 256 correlated noise
samples per coil (condition number 50), lambda 0.005, 120 iterations -- for
one slice, through the whole CsRss pipeline (strategy.rs:782-891), with the
readout-direction transforms of the FISTA loop on the FP32 SIMT FFT and on
the split-3xBF16 tensor-core DFT.  Both must reach NRMSE <= 1e-4 against the
FP64 oracle of the same pipeline; the values are printed (pytest -s)."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import strategy_ref
from openkspace_b200 import synth
from openkspace_b200.strategy import CsRss, oversampled_acquisitions

pytestmark = pytest.mark.gpu


def test_precision_slice_simt_vs_tensor_core_dft(ctx):
    vol = synth.oversampled_volume(nz=1)
    a = oversampled_acquisitions(vol)
    s = CsRss(iters=120, lambda_=0.005)
    want = strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                          iters=120, lam=0.005, remove_oversampling=True, prewhiten=True,
                                          fft_mode="auto", crop=True)
    got = {}
    try:
        for engine in (0, 1):
            ctx.set_option("row_engine", engine)
            got[engine] = s.reconstruct(ctx, a).data
    finally:
        ctx.set_option("row_engine", 0)
    assert ctx.tc_status() == 0
    e_simt, e_tc = o64.nrmse(got[0], want), o64.nrmse(got[1], want)
    print(f"\nprecision slice NRMSE vs FP64: SIMT FFT {e_simt:.3e}, tensor-core 3xBF16 DFT {e_tc:.3e}")
    assert got[0].shape == want.shape == (1, 368, 320)
    assert e_simt <= 1e-4
    assert e_tc <= 1e-4
    assert np.isfinite(got[1]).all()
