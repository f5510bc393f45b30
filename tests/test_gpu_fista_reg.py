"""The register-resident column engine (k_fista_col_reg) against the generic
shared-memory engine and the FP64 oracle, for every column length it has a
compile-time plan for.  Tolerance: relative L2 <= 1e-4."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from openkspace_b200 import Context
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


def row_mask(rng, ny, nx, frac=0.35):
    rows = rng.random(ny) < frac
    rows[ny // 2 - 2:ny // 2 + 2] = True
    return np.repeat(rows[:, None], nx, axis=1)


@pytest.fixture(scope="module")
def ctx2():
    c = Context(0)
    yield c
    c.close()


def run(ctx, engine, k, m, iters, lam):
    ctx.check(ctx.lib.okscuda_set_option(ctx.handle, b"col_engine", engine))
    try:
        return ctx.fista_cs(k, m, iters, lam)
    finally:
        ctx.check(ctx.lib.okscuda_set_option(ctx.handle, b"col_engine", 0))


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("ny", [128, 192, 256, 320, 368, 384, 512])
def test_register_engine_matches(ctx2, rng, ny, variant):
    """Both plans where a length has two (col_variant 1: the E = 8 one)."""
    nx, nc, iters = 12, 3, 12
    m = row_mask(rng, ny, nx)
    k = np.where(m[None], crandn(rng, (nc, ny, nx)), 0).astype(np.complex64)
    ctx2.set_option("col_variant", variant)
    try:
        reg = run(ctx2, 2, k, m, iters, 0.05)
    finally:
        ctx2.set_option("col_variant", -1)
    gen = run(ctx2, 1, k, m, iters, 0.05)
    assert rel_l2(reg, gen) < 1e-5
    assert rel_l2(reg, o64.fista_cs_single_coil(k, m, iters, 0.05)) < TOL_CS


def test_register_engine_edges(ctx2, rng):
    ny, nx = 256, 6
    k = crandn(rng, (2, ny, nx))
    for m in (np.zeros((ny, nx), bool), np.ones((ny, nx), bool), row_mask(rng, ny, nx)):
        kz = np.where(m[None], k, 0).astype(np.complex64)
        for iters in (0, 1, 7):
            reg = run(ctx2, 2, kz, m, iters, 0.02)
            assert rel_l2(reg, o64.fista_cs_single_coil(kz, m, iters, 0.02)) < TOL_CS
    # many problems, odd number of column pairs (partial last CTA)
    m = row_mask(rng, ny, 10)
    kz = np.where(m[None], crandn(rng, (5, ny, 10)), 0).astype(np.complex64)
    assert rel_l2(run(ctx2, 2, kz, m, 9, 0.01), o64.fista_cs_single_coil(kz, m, 9, 0.01)) < TOL_CS


def test_register_engine_plain_workload(ctx2):
    from openkspace_b200 import synth
    s = synth.plain_slice(0)
    reg = run(ctx2, 2, s.kspace, s.mask2d, 50, 0.01)
    x64 = o64.fista_cs_single_coil(s.kspace, s.mask2d, 50, 0.01)
    assert o64.nrmse(o64.rss_combine(reg), o64.rss_combine(x64)) < TOL_CS
