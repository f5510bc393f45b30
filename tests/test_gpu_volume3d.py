"""The CsRss 3-D path at a reduced size of the 3-D Cartesian workload
(placement with kspace_encode_step_2, centred IFFT along kz, per-slice
FISTA, RSS, crop) against the FP64 pipeline oracle: NRMSE <= 1e-4."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import strategy_ref
from openkspace_b200 import synth
from openkspace_b200.strategy import CsRss, cartesian3d_acquisitions

pytestmark = pytest.mark.gpu


def test_cartesian3d_pipeline_matches_oracle(ctx):
    k, m = synth.volume_3d(nc=4, nz=12, ny=64, nx=48)
    a = cartesian3d_acquisitions(k, m)
    s = CsRss(iters=15, lambda_=0.01)
    got = s.reconstruct(ctx, a).data
    want = strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                          iters=15, lam=0.01)
    assert got.shape == want.shape == (12, 64, 48)
    assert o64.nrmse(got, want) < 1e-4
