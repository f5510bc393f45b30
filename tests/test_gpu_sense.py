"""SENSE extension mode against its FP64 oracle (oracle/sense_fp64.py):
Walsh maps (f32 on the device, like the reference) to 1e-4, the FP64 power
iteration to 1e-9 on the same maps, the SENSE FISTA image to NRMSE 1e-4."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import sense_fp64 as sref
from openkspace_b200 import synth
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


@pytest.mark.parametrize("ny,nx,nc", [(128, 24, 4), (256, 16, 6), (368, 12, 3)])
def test_sense_matches_oracle(ctx, ny, nx, nc):
    s = synth.make_slice(ny, nx, nc, 4.0, 16, seed=ny + nc)
    m = s.mask2d
    mag, x, maps, L = ctx.sense_cs(s.kspace, m, 15, 0.005, walsh_window=3, walsh_iters=6, power_iters=30)
    imgs = sref.lowres_images(s.kspace, s.mask_rows)
    want_maps = sref.normalise_maps(sref.walsh_maps(imgs, 3, 6))
    assert rel_l2(maps, want_maps) < 1e-4
    assert 0.5 < L <= 1.0 + 1e-6          # unit-RSS maps and a unitary F: ||A||^2 <= 1
    assert abs(L - sref.lipschitz(maps.astype(np.complex128), m, 30)) < 1e-9 * max(L, 1)
    want = sref.sense_fista(s.kspace, maps.astype(np.complex128), m, 15, 0.005, L)
    assert rel_l2(x, want) < TOL_CS
    assert o64.nrmse(mag, np.abs(want)) < TOL_CS


def test_sense_acs_block():
    rows = np.zeros(32, bool)
    rows[[1, 3, 5]] = True
    rows[10:18] = True
    rows[20:23] = True
    assert sref.acs_rows(rows) == (10, 18)
    assert sref.acs_rows(np.eye(1, 32, 3, dtype=bool)[0]) is None
