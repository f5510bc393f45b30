"""The bounds-checked build (libokscuda_bounds.so: the same sources with
-DOKS_BOUNDS_CHECK) on small parity cases of every register-resident kernel
form: the standalone row and column transforms of every plan length (tiles
of 2, 4, 8 column pairs and every lanes form), the column FISTA engine on both
plans of every length, the 2-D-mask engine's register passes in each launch
form (plain, pipelined column and row passes, both register budgets) and the
SENSE engine.  Every exchange-buffer and staging index is range-checked in
that build; the error word (okscuda_debug_bounds) must stay 0, and every
result must still match the FP64 oracle.  Runs in a child process that loads
the checked library (OKSCUDA_LIB=bounds)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from openkspace_b200 import Context, synth
from oracle import cs_fp64 as o64
rng = np.random.default_rng(5)
def crandn(shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-30))
out = {"errors": [], "word": None}
with Context(0) as ctx:
    assert b"bounds-checked" in ctx.lib.okscuda_version()
    w = ctypes.c_uint()
    ctx.check(ctx.lib.okscuda_debug_bounds(ctx.handle, ctypes.byref(w), 1))   # start from 0
    lengths = [128, 192, 256, 320, 368, 384, 512, 640]
    for n in lengths:                                   # rows and columns, both directions
        x = crandn((2, n, 40 if n != 368 else 20))
        for inv in (False, True):
            got = ctx.centred_fft2(x, inv)
            want = o64.centred_ifft2(x) if inv else o64.centred_fft2(x)
            if rel(got, want) > 1e-5:
                out["errors"].append(f"fft2 {n} inv={inv}")
        lanes_forms = {368: (5, 6, 7, 8, 9), 640: (1, 2, 3, 4, 10), 320: (1, 2, 3, 4, 11)}.get(n, (1, 2, 3, 4))
        for opt, vals in (("xform_tile", (2, 4, 8)), ("xform_lanes", lanes_forms)):
            for v in vals:
                for pf in ((0, 1) if opt == "xform_lanes" else (0,)):
                    ctx.set_option(opt, v)
                    ctx.set_option("xform_lanes_pf", pf)
                    got = ctx.centred_fft2(x, True)
                    ctx.set_option(opt, 0)
                    ctx.set_option("xform_lanes_pf", 1)
                    if rel(got, o64.centred_ifft2(x)) > 1e-5:
                        out["errors"].append(f"fft2 {n} {opt}={v} pf={pf}")
    for nr in (368, 320):                               # two-stage and register-tile row forms
        xr = crandn((2, 22, nr))
        for var in (0, 3, 1):
            ctx.set_option("xform_row_variant", var)
            for inv in (False, True):
                got = ctx.centred_fft2(xr, inv)
                want = o64.centred_ifft2(xr) if inv else o64.centred_fft2(xr)
                if rel(got, want) > 1e-5:
                    out["errors"].append(f"fft2 rows {nr} variant={var} inv={inv}")
    ctx.set_option("xform_row_variant", 0)
    for n in (128, 192, 256, 320, 368, 384, 512):       # column engine, both plans
        rows = rng.random(n) < 0.35
        rows[n // 2 - 2:n // 2 + 2] = True
        m = np.repeat(rows[:, None], 12, axis=1)
        k = np.where(m[None], crandn((2, n, 12)), 0).astype(np.complex64)
        want = o64.fista_cs_single_coil(k, m, 6, 0.02)
        for var in (0, 1):
            ctx.set_option("col_variant", var)
            got = ctx.fista_cs(k, m, 6, 0.02)
            ctx.set_option("col_variant", -1)
            if o64.nrmse(got, want) > 1e-4:
                out["errors"].append(f"column engine {n} variant {var}")
    forms = [dict(occ2d=1, prefetch2d=1), dict(occ2d=1, prefetch2d=0), dict(occ2d=1, prefetch2d=3),
             dict(occ2d=2, prefetch2d=3), dict(occ2d=0, prefetch2d=0, persist2d=0), dict(occ2d=1, prefetch2d=5),
             dict(occ2d=0, prefetch2d=4, persist2d=0), dict(col2d_lanes=5), dict(col2d_lanes=6), dict(col2d_lanes=7), dict(col2d_lanes=8), dict(col2d_lanes=1),
             dict(col2d_lanes=3), dict(col2d_lanes=-1), dict(col2d_lanes=9),
             dict(col2d_lanes=10), dict(col2d_lanes=11), dict(col2d_lanes=12),
             dict(col2d_lanes=13), dict(col2d_lanes=14)]
    default = dict(occ2d=1, prefetch2d=1, persist2d=1, col2d_lanes=0)
    for ny, nx in ((368, 640), (256, 192), (384, 320), (128, 512)):   # 2-D engine, partial rows
        m = np.zeros((ny, nx), bool)
        m[rng.random(ny) < 0.3, nx // 4: 3 * nx // 4] = True
        m[ny // 2, :] = True
        k = np.where(m[None], crandn((3, ny, nx)), 0).astype(np.complex64)
        want = o64.fista_cs_single_coil(k, m, 3, 0.02)
        for f in forms:
            for a, v in f.items():
                ctx.set_option(a, v)
            got = ctx.fista_cs(k, m, 3, 0.02)
            for a, v in default.items():
                ctx.set_option(a, v)
            if o64.nrmse(got, want) > 1e-4:
                out["errors"].append(f"2-D engine {ny}x{nx} {f}")
    from oracle import sense_fp64 as sref
    s = synth.make_slice(128, 24, 4, 4.0, 12, seed=7)        # SENSE engine
    mag, x, maps, L = ctx.sense_cs(s.kspace, s.mask2d, 5, 0.01)
    want = sref.sense_fista(s.kspace, maps.astype(np.complex128), s.mask2d, 5, 0.01, L)
    if rel(x, want) > 1e-4:
        out["errors"].append("sense")
    ctx.check(ctx.lib.okscuda_debug_bounds(ctx.handle, ctypes.byref(w), 1))
    out["word"] = w.value
print("RESULT " + json.dumps(out))
"""


def test_bounds_checked_build_small_cases():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, OKSCUDA_LIB="bounds")
    p = subprocess.run([sys.executable, "-c", _CHILD, root], env=env, capture_output=True, text=True, timeout=1200)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    line = next(ln for ln in p.stdout.splitlines() if ln.startswith("RESULT "))
    out = json.loads(line[len("RESULT "):])
    assert out["word"] == 0, out
    assert out["errors"] == [], out


def test_normal_build_reports_not_bounds_checked(ctx):
    import ctypes

    from openkspace_b200 import _lib
    w = ctypes.c_uint(7)
    assert ctx.lib.okscuda_debug_bounds(ctx.handle, ctypes.byref(w), 0) == _lib.OKS_ENOTSUP
    assert w.value == 0
