"""Request server: every result in a mix of concurrent requests equals the
same request solved alone (NRMSE <= 1e-4, in practice bit-identical kernels),
admission refuses what does not fit, waits are bounded."""
import time

import numpy as np
import pytest

from oracle import cs_fp64 as o64
from openkspace_b200 import OksError, _lib, synth
from openkspace_b200.server import Server
from tests.conftest import crandn

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


@pytest.mark.parametrize("mode", [0, 1])
def test_mix_equals_alone(ctx, mode):
    """Mode 0 runs one chain per request, mode 1 merges the queued requests
    into batched passes: every result equals the request solved alone."""
    reqs = synth.uneven_requests(n=12, sizes=((256, 256), (320, 320), (368, 64), (64, 48)), coil_range=(2, 6),
                                 iter_range=(5, 25))
    masks = [np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1) for r in reqs]
    alone = [ctx.cs_slice(r.kspace, m, r.iters, r.lam) for r, m in zip(reqs, masks)]
    with Server(ctx, max_inflight=8, n_streams=4, mode=mode) as srv:
        pending = list(range(len(reqs)))
        ids = {}
        while pending:                       # submit everything, resubmitting refused requests
            i = pending[0]
            try:
                ids[i] = srv.submit(reqs[i].kspace, masks[i], reqs[i].iters, reqs[i].lam)
                pending.pop(0)
            except OksError as e:
                assert e.code == _lib.OKS_EAGAIN
                time.sleep(0.001)
        for i, (rid, out) in ids.items():
            srv.wait(rid, 60000)
            assert o64.nrmse(out, alone[i]) < TOL_CS
        assert srv.stats()["inflight"] == 0


def test_admission_by_budget(ctx, rng):
    k = crandn(rng, (4, 64, 64))
    m = np.ones((64, 64), bool)
    need = 4 * 64 * 64 * 8 * 4 + 64 * 64 * 4
    with Server(ctx, max_inflight=4, hbm_budget_bytes=need + 10) as srv:
        rid, out = srv.submit(k, m, 20000, 0.01)   # long enough to still run below
        with pytest.raises(OksError) as e:
            srv.submit(k, m, 5, 0.01)        # budget holds one request
        assert e.value.code == _lib.OKS_EAGAIN
        srv.wait(rid, 120000)
        rid2, out2 = srv.submit(k, m, 20000, 0.01)   # admitted once memory is back
        srv.wait(rid2, 120000)
        assert np.array_equal(out, out2)


def test_wait_timeout_is_bounded(ctx, rng):
    k = crandn(rng, (8, 256, 256))
    m = np.ones((256, 256), bool)
    with Server(ctx) as srv:
        rid, out = srv.submit(k, m, 3000, 0.01)
        with pytest.raises(OksError) as e:
            srv.wait(rid, 0)
        assert e.value.code == _lib.OKS_ETIMEDOUT
        srv.wait(rid, 120000)


def test_device_resident_request(ctx, rng):
    s = synth.make_slice(64, 32, 3, 4.0, 8, seed=5)
    d = ctx.to_device(s.kspace)
    with Server(ctx) as srv:
        rid, out = srv.submit(None, s.mask2d, 20, 0.01, device=d)
        srv.wait(rid, 60000)
    assert o64.nrmse(out, ctx.cs_slice(s.kspace, s.mask2d, 20, 0.01)) < 1e-6
    assert np.array_equal(d.to_host(), s.kspace)   # input left untouched


@pytest.mark.parametrize("mode", [0, 1])
def test_volume_slices_in_place_and_2d_masks(ctx, mode):
    """Slices of a device-resident [nc, nz, ny, nx] volume submitted in place
    (coil planes nz * ny * nx apart), a 2-D (partial-row) mask request in the
    same batch, and a pageable output: each equals the slice solved alone."""
    rng = np.random.default_rng(3)
    nc, nz, ny, nx = 3, 4, 64, 48
    rows = rng.random(ny) < 0.4
    rows[ny // 2 - 3:ny // 2 + 3] = True
    m = np.repeat(rows[:, None], nx, 1)
    vol = np.where(m[None, None], crandn(rng, (nc, nz, ny, nx)), 0).astype(np.complex64)
    d = ctx.to_device(vol)
    m2 = m.copy()
    m2[:, :8] = False                                   # rows partial in kx: the 2-D engine
    k2 = np.where(m2[None], crandn(rng, (2, ny, nx)), 0).astype(np.complex64)
    with Server(ctx, mode=mode) as srv:
        ids = [srv.submit(None, m, 12, 0.01, device_slice=(d, z)) for z in range(nz)]
        i2 = srv.submit(k2, m2, 9, 0.02)
        for rid, _ in ids + [i2]:
            srv.wait(rid, 60000)
    for z, (_, out) in enumerate(ids):
        assert o64.nrmse(out, ctx.cs_slice(np.ascontiguousarray(vol[:, z]), m, 12, 0.01)) < 1e-6
    assert o64.nrmse(i2[1], ctx.cs_slice(k2, m2, 9, 0.02)) < 1e-6
    assert np.array_equal(d.to_host(), vol)             # the volume is left untouched
