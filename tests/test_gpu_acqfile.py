"""Configuration-1 ingest: one slice of the precision workload written as an
acquisition stream file, read back through okscuda_raw_open (samples in a
pinned buffer) and reconstructed by the CsRss pipeline: bit-identical to the
reconstruction of the in-memory set, and within 1e-4 of the FP64 oracle."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import strategy_ref
from openkspace_b200 import synth
from openkspace_b200.acqfile import read_acquisitions, write_acquisitions
from openkspace_b200.strategy import CsRss, oversampled_acquisitions

pytestmark = pytest.mark.gpu


def test_file_reconstruction_equals_in_memory(ctx, tmp_path):
    vol = synth.oversampled_volume(nz=1)
    a = oversampled_acquisitions(vol)
    s = CsRss(iters=30, lambda_=0.005)
    want = s.reconstruct(ctx, a).data
    p = str(tmp_path / "precision_slice0.oksacq")
    write_acquisitions(p, a, receiver_channels=vol.lines.shape[2])
    with read_acquisitions(p) as f:
        got = s.reconstruct(ctx, f.acqs).data
    assert np.array_equal(got, want)
    ref = strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                         iters=30, lam=0.005, workers=8)
    assert o64.nrmse(got, ref) < 1e-4
