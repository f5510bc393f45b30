"""okscuda_cs_batch: slices of uneven size, coil count, iteration count,
lambda and mask solved together must equal each slice solved alone (and the
FP64 oracle) -- NRMSE <= 1e-4."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from openkspace_b200 import synth
from tests.conftest import crandn

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


def make(rng, ny, nx, nc, iters, lam, kind="rows"):
    rows = rng.random(ny) < 0.35
    rows[ny // 2 - 2:ny // 2 + 2] = True
    m = np.repeat(rows[:, None], nx, axis=1)
    if kind == "partial":
        m[:, : nx // 4] = False
    k = np.where(m[None], crandn(rng, (nc, ny, nx)), 0).astype(np.complex64)
    return k, m, iters, lam


def test_batch_uneven_matches_alone_and_oracle(ctx, rng):
    sl = [make(rng, 256, 16, 3, 20, 0.02), make(rng, 320, 12, 2, 7, 0.05), make(rng, 368, 20, 4, 15, 0.01),
          make(rng, 256, 8, 1, 0, 0.01), make(rng, 384, 10, 2, 11, 0.03), make(rng, 40, 12, 2, 9, 0.02),
          make(rng, 24, 16, 2, 6, 0.02, kind="partial"), make(rng, 256, 16, 2, 25, 0.001)]
    got = ctx.cs_batch(sl)
    for (k, m, iters, lam), g in zip(sl, got):
        alone = ctx.cs_slice(k, m, iters, lam)
        assert o64.nrmse(g, alone) < 1e-6
        want = o64.rss_combine(o64.fista_cs_single_coil(k, m, iters, lam))
        assert o64.nrmse(g, want) < TOL_CS


def test_batch_generated_requests(ctx):
    reqs = synth.uneven_requests(n=6, sizes=((256, 256), (320, 320)), coil_range=(2, 4), iter_range=(5, 12))
    got = ctx.cs_batch([(r.kspace, np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1), r.iters, r.lam)
                        for r in reqs])
    for r, g in zip(reqs, got):
        m = np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1)
        want = o64.rss_combine(o64.fista_cs_single_coil(r.kspace, m, r.iters, r.lam))
        assert o64.nrmse(g, want) < TOL_CS


def test_batch_empty_and_errors(ctx, rng):
    assert ctx.cs_batch([]) == []
    from openkspace_b200 import OksError, _lib
    with pytest.raises(OksError) as e:
        ctx.cs_batch([(np.zeros((1, 7, 8), np.complex64), np.ones((7, 8), bool), 3, 0.01)])
    assert e.value.code == _lib.OKS_EODD
