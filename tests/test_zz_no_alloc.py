"""okscuda_cs_slice_noalloc: the allocation-free per-slice entry point for
callers whose device memory is owned by their own allocator and who may not
call cudaMalloc.  Called through the C-ABI; checked against okscuda_cs_slice
(the entry point that allocates its scratch) on two calls in a row, within the
tolerance of the other FISTA-CS parity tests (relative L2 1e-4).  Collected
last so that a failure here leaves every other test already run."""
import ctypes
import json
import os
import subprocess
import sys

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


# Child process: the allocation counter (tests/support/alloc_counter.c) is
# preloaded, so every cudaMalloc / cudaMallocAsync / cudaMallocHost / cudaFree
# ... that libokscuda.so makes is counted.  The first call of the entry point
# in the process, at a row length whose register transform has never run
# (the library would build that plan's tables on first use), and a second
# call at another length, must make none; the allocating entry point then
# gives the reference result.
_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
probe = ctypes.CDLL(None)
from openkspace_b200 import Context, synth
out = {}
with Context(0) as ctx:
    L = ctx.lib
    p = ctypes.c_void_p()
    probe.oks_alloc_probe_reset()
    ctx.check(L.okscuda_malloc(ctx.handle, 256, ctypes.byref(p)))
    out["control"] = probe.oks_alloc_probe_count()      # the counter sees the library's calls
    ctx.check(L.okscuda_free(ctx.handle, p))
    shapes = [(256, 256, 4, 30, 11), (320, 320, 3, 20, 12)]
    res = []
    for ny, nx, nc, iters, seed in shapes:
        sl = synth.make_slice(ny, nx, nc, 4.0, 24, seed=seed)
        k = np.ascontiguousarray(sl.kspace)
        m = np.ascontiguousarray(sl.mask2d, dtype=np.uint8)
        d_k = ctx.to_device(k)
        got = ctx.empty((ny, nx), np.float32)
        ctx.synchronize()
        probe.oks_alloc_probe_reset()
        ctx.check(L.okscuda_cs_slice_noalloc(ctx.handle, d_k.ptr, m.ctypes.data, nc, ny, nx, iters,
                                             ctypes.c_float(0.01), got.ptr))
        ctx.synchronize()
        res.append({"allocs": probe.oks_alloc_probe_count(), "got": got.to_host()})
        want = ctx.empty((ny, nx), np.float32)
        ctx.check(L.okscuda_cs_slice(ctx.handle, d_k.ptr, m.ctypes.data, nc, ny, nx, iters,
                                     ctypes.c_float(0.01), want.ptr, None))
        res[-1]["want"] = want.to_host()
    for r in res:
        g, w = r["got"].ravel(), r["want"].ravel()
        r["rel"] = float(np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-30))
        del r["got"], r["want"]
    out["calls"] = res
print("RESULT " + json.dumps(out))
"""


def test_noalloc_first_call_allocates_nothing(tmp_path):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    shim = tmp_path / "alloc_counter.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O2", os.path.join(root, "tests", "support", "alloc_counter.c"),
                    "-o", str(shim), "-ldl"], check=True)
    env = dict(os.environ, LD_PRELOAD=str(shim))
    p = subprocess.run([sys.executable, "-c", _CHILD, root], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    line = next(ln for ln in p.stdout.splitlines() if ln.startswith("RESULT "))
    out = json.loads(line[len("RESULT "):])
    assert out["control"] >= 1, "the allocation counter did not see okscuda_malloc"
    for c in out["calls"]:
        assert c["allocs"] == 0, out
        assert c["rel"] < TOL_CS, out
