"""okscuda_cs_slice_noalloc: the allocation-free per-slice entry point for
callers whose device memory is owned by their own allocator and who may not
call cudaMalloc.  Called through the C-ABI; checked against okscuda_cs_slice
(the entry point that allocates its scratch) on two calls in a row, within the
tolerance of the other FISTA-CS parity tests (relative L2 1e-4).  Collected
last so that a failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

from openkspace_b200 import Context, _lib, synth
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4


def _slice_both(ctx, sl, iters, lam):
    k = np.ascontiguousarray(sl.kspace)
    nc, ny, nx = k.shape
    m = np.ascontiguousarray(sl.mask2d, dtype=np.uint8)
    d_k = ctx.to_device(k)
    want = ctx.empty((ny, nx), np.float32)
    got = ctx.empty((ny, nx), np.float32)
    L = ctx.lib
    ctx.check(L.okscuda_cs_slice(ctx.handle, d_k.ptr, m.ctypes.data, nc, ny, nx, iters, ctypes.c_float(lam),
                                 want.ptr, None))
    ctx.check(L.okscuda_cs_slice_noalloc(ctx.handle, d_k.ptr, m.ctypes.data, nc, ny, nx, iters,
                                         ctypes.c_float(lam), got.ptr))
    return got.to_host(), want.to_host()


def test_noalloc_matches_allocating_entry_point_twice():
    with Context(0) as ctx:
        # two calls in a row with different shapes, masks and iteration counts:
        # the second call must not see anything the first left in the array
        a = synth.make_slice(64, 48, 4, 4.0, 12, seed=101)
        got, want = _slice_both(ctx, a, 30, 0.01)
        assert np.all(np.isfinite(got))
        assert rel_l2(got, want) < TOL_CS
        b = synth.plain_slice(3)
        got2, want2 = _slice_both(ctx, b, 50, 0.01)
        assert rel_l2(got2, want2) < TOL_CS


def test_noalloc_rejects_sizes_beyond_its_array():
    with Context(0) as ctx:
        ny, nx, nc = 512, 512, 8          # 16 MiB of coil images: above the fixed array
        m = np.ones((ny, nx), np.uint8)
        d_k = ctx.empty((nc, ny, nx))
        out = ctx.empty((ny, nx), np.float32)
        rc = ctx.lib.okscuda_cs_slice_noalloc(ctx.handle, d_k.ptr, m.ctypes.data, nc, ny, nx, 5,
                                              ctypes.c_float(0.01), out.ptr)
        assert rc == _lib.OKS_ENOTSUP
        assert "scratch" in ctx.last_error()
