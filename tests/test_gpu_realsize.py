"""Parity at the benchmark configurations' real sizes (the other GPU tests
use reduced shapes): every result against the FP64 oracle at NRMSE <= 1e-4
on the RSS magnitude image.

* configuration 2: okscuda_cs_batch on slices of 384 x 384 and 368 x 640 (and
  256^2, 320^2) with 8-32 coils, iterations cut to 20-30 so that the FP64
  oracle finishes in seconds;
* configuration 3: the request server on a mix drawn from the serving
  distribution (sizes {256^2, 320^2, 384^2, 368 x 640}, coils U{8..32},
  R {2,3,4,6}); each result equals the same request solved alone, and the
  two largest are checked against the oracle;
* configuration 4: a 32-coil 256 x 256 x 8 (kz) sub-volume of the 3-D
  Cartesian workload (ky-only R = 6 + 24 centre lines, 80 iterations)
  through the CsRss 3-D path (kz IFFT, per-slice FISTA, RSS)."""
import os
import time

import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import strategy_ref
from openkspace_b200 import OksError, _lib, synth
from openkspace_b200.server import Server
from openkspace_b200.strategy import CsRss, cartesian3d_acquisitions

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4
WORKERS = os.cpu_count() or 1


def _oracle_rss(kspace, mask2d, iters, lam):
    return o64.csrss_from_kspace(kspace[:, None], mask2d[None], iters, lam, workers=WORKERS)[0]


def test_batch_config2_real_shapes(ctx):
    shapes = [(384, 384, 24, 2.0, 25), (368, 640, 32, 4.0, 20), (320, 320, 8, 6.0, 30), (256, 256, 16, 3.0, 30),
              (368, 640, 9, 2.0, 22)]
    slices = []
    for i, (ny, nx, nc, r, iters) in enumerate(shapes):
        s = synth.make_slice(ny, nx, nc, r, 24, seed=2000 + i)
        slices.append((s.kspace, s.mask2d, iters, 0.01))
    got = ctx.cs_batch(slices)
    for (k, m, iters, lam), g in zip(slices, got):
        want = _oracle_rss(k, m, iters, lam)
        err = o64.nrmse(g, want)
        assert err < TOL_CS, (k.shape, iters, err)


def test_server_mix_serving_distribution(ctx):
    reqs = synth.uneven_requests(n=10, workload=3, iter_range=(15, 30))
    masks = [np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1) for r in reqs]
    alone = [ctx.cs_slice(r.kspace, m, r.iters, r.lam) for r, m in zip(reqs, masks)]
    with Server(ctx, max_inflight=16, n_streams=8) as srv:
        ids = {}
        pending = list(range(len(reqs)))
        while pending:                       # all submitted at once: they overlap on the device
            i = pending[0]
            try:
                ids[i] = srv.submit(reqs[i].kspace, masks[i], reqs[i].iters, reqs[i].lam)
                pending.pop(0)
            except OksError as e:
                assert e.code == _lib.OKS_EAGAIN
                time.sleep(0.001)
        for i, (rid, out) in ids.items():
            srv.wait(rid, 120000)
            assert o64.nrmse(out, alone[i]) < 1e-6, i
    order = sorted(range(len(reqs)), key=lambda i: -reqs[i].kspace.size)
    for i in order[:2]:
        r = reqs[i]
        want = _oracle_rss(r.kspace, masks[i], r.iters, r.lam)
        assert o64.nrmse(ids[i][1], want) < TOL_CS, (r.kspace.shape, r.iters)


def test_cartesian3d_subvolume_32_coils(ctx):
    k, m = synth.volume_3d(nc=32, nz=8, ny=256, nx=256)
    a = cartesian3d_acquisitions(k, m)
    s = CsRss(iters=80, lambda_=0.01)
    got = s.reconstruct(ctx, a).data
    want = strategy_ref.csrss_reconstruct(a.headers, a.data, a.encoded, a.recon, a.ky_center, a.kz_center,
                                          iters=80, lam=0.01, workers=WORKERS)
    assert got.shape == want.shape == (8, 256, 256)
    assert o64.nrmse(got, want) < TOL_CS


@pytest.mark.parametrize("mode", [0, 1])
def test_cartesian3d_slices_through_the_server(ctx, mode):
    """Configuration 4's path through the request server: the kz-decoupled
    32-coil 256 x 256 x 8 volume's slices submitted in place, back to back,
    under an HBM budget that holds 2.5 of them (so admission refuses some),
    then serving requests beside them; each slice equals the CsRss 3-D
    path's slice, and each serving request its result alone."""
    from openkspace_b200 import Context
    k, m = synth.volume_3d(nc=32, nz=8, ny=256, nx=256)
    want = CsRss(iters=80, lambda_=0.01).reconstruct(ctx, cartesian3d_acquisitions(k, m)).data
    reqs = synth.uneven_requests(n=4, workload=3, sizes=((256, 256), (320, 320)), coil_range=(8, 12),
                                 iter_range=(15, 25))
    masks = [np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1) for r in reqs]
    alone = [ctx.cs_slice(r.kspace, mk, r.iters, r.lam) for r, mk in zip(reqs, masks)]
    nc, nz, ny, nx = k.shape
    slice_need = 4 * nc * ny * nx * 8 + ny * nx * 4          # work copy + RSS + worst-case 2-D scratch
    refused = 0
    with Context(0) as sctx:
        d = sctx.to_device(k)
        sctx.check(sctx.lib.okscuda_ifft1_kz(sctx.handle, d.ptr, nc, nz, ny, nx))
        m2 = np.repeat(m[:, None], nx, 1)
        with Server(sctx, max_inflight=16, hbm_budget_bytes=int(2.5 * slice_need), mode=mode) as srv:
            ids, sids = [], []
            todo = [("v", z) for z in range(nz)] + [("r", i) for i in range(len(reqs))]
            for kind, i in todo:
                while True:
                    try:
                        if kind == "v":
                            ids.append((i, srv.submit(None, m2, 80, 0.01, device_slice=(d, i))))
                        else:
                            sids.append((i, srv.submit(reqs[i].kspace, masks[i], reqs[i].iters, reqs[i].lam)))
                        break
                    except OksError as e:
                        assert e.code == _lib.OKS_EAGAIN
                        refused += 1
                        time.sleep(0.0005)
            for _, (rid, _) in ids + sids:
                srv.wait(rid, 120000)
    assert refused > 0                                   # the budget did push back
    for z, (_, out) in ids:
        assert o64.nrmse(out, want[z]) < 1e-6, z
    for i, (_, out) in sids:
        assert o64.nrmse(out, alone[i]) < 1e-6, i
