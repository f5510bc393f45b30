"""Register-resident centred transforms (k_row_xform_reg / k_col_xform_reg)
through the C-ABI, against the FP64 centred FFT of cs.rs:141-218 (shifts of
shift.rs:11-26) and against the shared-memory kernels they replace.

Tolerance: relative L2 1e-5 for single FP32 transforms (the bound of the
other primitive tests); the two FP32 engines agree to the same bound.
"""
import ctypes

import numpy as np
import pytest

from oracle import cs_fp64 as o64
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
LENGTHS = [128, 192, 256, 320, 368, 384, 512, 640]


def ref_rows(x, inverse, centred):
    a = x.astype(np.complex128)
    if centred:
        a = o64.ifftshift_axis(a, -1)
    a = np.fft.ifft(a, axis=-1) * a.shape[-1] if inverse else np.fft.fft(a, axis=-1)
    if centred:
        a = o64.fftshift_axis(a, -1)
    return a


def both_engines(ctx, fn):
    out = {}
    try:
        for eng in (0, 1):
            ctx.set_option("xform_engine", eng)
            out[eng] = fn()
    finally:
        ctx.set_option("xform_engine", 1)
    return out[0], out[1]


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("inverse", [False, True])
def test_centred_fft2_every_plan_length(ctx, rng, n, inverse):
    """Rows and columns of every register plan length, both directions."""
    x = crandn(rng, (2, n, n if n <= 384 else 96))
    gen, reg = both_engines(ctx, lambda: ctx.centred_fft2(x, inverse))
    want = o64.centred_ifft2(x) if inverse else o64.centred_fft2(x)
    assert rel_l2(reg, want) < TOL
    assert rel_l2(gen, want) < TOL
    assert rel_l2(reg, gen) < TOL


@pytest.mark.parametrize("ny,nx", [(368, 640), (640, 368), (256, 100), (320, 18), (512, 2), (128, 30),
                                   (192, 75), (384, 7)])
@pytest.mark.parametrize("inverse", [False, True])
def test_centred_fft2_ragged_tiles(ctx, rng, ny, nx, inverse):
    """Column counts that leave a partial tile (and odd ones, which take the
    shared-memory column kernel while the rows stay on the register kernel)."""
    x = crandn(rng, (3, ny, nx))
    _, reg = both_engines(ctx, lambda: ctx.centred_fft2(x, inverse))
    want = o64.centred_ifft2(x) if inverse else o64.centred_fft2(x)
    assert rel_l2(reg, want) < TOL


@pytest.mark.parametrize("tile", [2, 4, 8])
@pytest.mark.parametrize("ny", [256, 368, 512, 640])
def test_column_tile_widths(ctx, rng, tile, ny):
    x = crandn(rng, (2, ny, 48))
    want = o64.centred_fft2(x)
    ctx.set_option("xform_tile", tile)
    try:
        got = ctx.centred_fft2(x)
    finally:
        ctx.set_option("xform_tile", 0)
    assert rel_l2(got, want) < TOL


@pytest.mark.parametrize("lanes", [-1, 1, 2, 3, 4])
@pytest.mark.parametrize("n", LENGTHS)
def test_column_lanes_forms(ctx, rng, n, lanes):
    """Every (tile width, threads per column) form of the lanes-across-columns
    kernel, and the tiles (lanes -1), on ragged column counts."""
    x = crandn(rng, (2, n, 38 if n != 368 else 20))
    want = o64.centred_ifft2(x)
    ctx.set_option("xform_lanes", lanes)
    try:
        got = ctx.centred_fft2(x, True)
    finally:
        ctx.set_option("xform_lanes", 0)
    assert rel_l2(got, want) < TOL


@pytest.mark.parametrize("pf", [0, 1])
@pytest.mark.parametrize("lanes", [1, 2, 3, 4])
@pytest.mark.parametrize("n", [n for n in LENGTHS if n != 368])
def test_column_lanes_pipelined_and_direct(ctx, rng, n, lanes, pf):
    """The lanes form, software-pipelined (next tile staged in shared memory
    with cp.async, the default) and direct: several tiles per CTA, a ragged
    last tile, both directions, and an odd column count (which always takes
    the direct form)."""
    for ncols, inverse in ((38, True), (130, False), (7, True)):
        x = crandn(rng, (3, n, ncols))
        want = o64.centred_ifft2(x) if inverse else o64.centred_fft2(x)
        ctx.set_option("xform_lanes", lanes)
        ctx.set_option("xform_lanes_pf", pf)
        try:
            got = ctx.centred_fft2(x, inverse)
        finally:
            ctx.set_option("xform_lanes", 0)
            ctx.set_option("xform_lanes_pf", 1)
        assert rel_l2(got, want) < TOL


@pytest.mark.parametrize("rows,n", [(1, 640), (301, 368), (7, 128), (1001, 320), (64, 512)])
@pytest.mark.parametrize("inverse,centred", [(0, 1), (1, 1), (0, 0), (1, 0)])
def test_rows_odd_counts_and_uncentred(ctx, rng, rows, n, inverse, centred):
    x = crandn(rng, (rows, n))
    gen, reg = both_engines(ctx, lambda: ctx.dft_rows(x, inverse=bool(inverse), centred=bool(centred), engine=0))
    want = ref_rows(x, inverse, centred)
    assert rel_l2(reg, want) < TOL
    assert rel_l2(gen, want) < TOL


def test_rows_in_place(ctx, rng):
    x = crandn(rng, (77, 384))
    got = ctx.dft_rows(x, inverse=True, centred=True, engine=0, in_place=True)
    assert rel_l2(got, ref_rows(x, 1, 1)) < TOL


def test_rows_unaligned_input(ctx, rng):
    """Rows that start 8 bytes off a 16-byte boundary take the 8-byte copies."""
    rows, n = 45, 256
    x = crandn(rng, (rows * n + 1,))
    d = ctx.to_device(x)
    o = ctx.empty((rows, n))
    ctx.check(ctx.lib.okscuda_dft_rows(ctx.handle, ctypes.c_void_p(d.ptr + 8), o.ptr, rows, n, 0, 1, 0))
    got = o.to_host()
    assert rel_l2(got, ref_rows(x[1:].reshape(rows, n), 0, 1)) < TOL


def test_fista_prep_rows_same_on_both_engines(ctx, rng):
    """The column engine's prep (row IDFT with a ky row mask, row signs and
    scale) through both transform kernels: same reconstruction."""
    ny, nx = 368, 320
    rows = rng.random(ny) < 0.35
    rows[ny // 2 - 4:ny // 2 + 4] = True
    m = np.repeat(rows[:, None], nx, axis=1)
    k = np.where(m[None], crandn(rng, (2, ny, nx)), 0).astype(np.complex64)
    gen, reg = both_engines(ctx, lambda: ctx.fista_cs(k, m, 20, 0.01))
    want = o64.fista_cs_single_coil(k, m, 20, 0.01)
    assert o64.nrmse(reg, want) < 1e-4
    assert o64.nrmse(reg, gen) < 1e-5


@pytest.mark.parametrize("n,variant", [(192, 1), (192, 2), (320, 1), (368, 3), (320, 3)])
def test_row_plan_variants(ctx, rng, n, variant):
    """The alternative register row plans (option xform_row_variant)."""
    x = crandn(rng, (3, 40, n))
    ctx.set_option("xform_row_variant", variant)
    try:
        got = ctx.centred_fft2(x, False)
        got_i = ctx.dft_rows(x.reshape(-1, n), inverse=True, centred=True, engine=0)
    finally:
        ctx.set_option("xform_row_variant", 0)
    assert rel_l2(got, o64.centred_fft2(x)) < TOL
    assert rel_l2(got_i, ref_rows(x.reshape(-1, n), 1, 1)) < TOL


def test_row_q368_ragged_and_in_the_column_engine(ctx, rng):
    """The two-stage 368 row transform (xform_row_variant 3): a row count that
    leaves a ragged last tile, both directions, and the column engine's
    readout pass (rows outside the ky mask kept at zero, per-problem row
    signs) under FISTA with a ky-only mask, against FP64."""
    x = crandn(rng, (61, 368))
    ctx.set_option("xform_row_variant", 3)
    try:
        got_f = ctx.dft_rows(x, inverse=False, centred=True, engine=0)
        got_i = ctx.dft_rows(x, inverse=True, centred=True, engine=0)
        ny, nx, iters = 256, 368, 6
        m = np.zeros((ny, nx), bool)
        m[rng.random(ny) < 0.3] = True
        m[ny // 2 - 4:ny // 2 + 4] = True
        k = np.where(m[None], crandn(rng, (3, ny, nx)), 0).astype(np.complex64)
        got_cs = ctx.fista_cs(k, m, iters, 0.02)
    finally:
        ctx.set_option("xform_row_variant", 0)
    assert rel_l2(got_f, ref_rows(x, 0, 1)) < TOL
    assert rel_l2(got_i, ref_rows(x, 1, 1)) < TOL
    assert rel_l2(got_cs, o64.fista_cs_single_coil(k, m, iters, 0.02)) < 1e-4


@pytest.mark.parametrize("n,form", [(640, 10), (320, 11)])
def test_column_two_stage(ctx, rng, n, form):
    """The two-stage column transforms (xform_lanes 10: 640 = 20 · 32; 11:
    320 = 16 · 20): both directions, ragged tiles and an odd column count
    (which takes the default form)."""
    for ncols, inverse in ((38, True), (130, False), (7, True), (40, False), (24, True)):
        x = crandn(rng, (2, n, ncols))
        want = o64.centred_ifft2(x) if inverse else o64.centred_fft2(x)
        ctx.set_option("xform_lanes", form)
        try:
            got = ctx.centred_fft2(x, inverse)
        finally:
            ctx.set_option("xform_lanes", 0)
        assert rel_l2(got, want) < TOL


@pytest.mark.parametrize("pf", [0, 1])
@pytest.mark.parametrize("lanes", [5, 6, 7, 8, 9])
def test_column_lanes_368(ctx, rng, lanes, pf):
    """The 368-point lanes forms (16 threads per column, one per radix-23
    butterfly), pipelined and direct, ragged and odd column counts."""
    for ncols, inverse in ((38, True), (130, False), (7, True), (40, False), (130, True)):
        x = crandn(rng, (2, 368, ncols))
        want = o64.centred_ifft2(x) if inverse else o64.centred_fft2(x)
        ctx.set_option("xform_lanes", lanes)
        ctx.set_option("xform_lanes_pf", pf)
        try:
            got = ctx.centred_fft2(x, inverse)
        finally:
            ctx.set_option("xform_lanes", 0)
            ctx.set_option("xform_lanes_pf", 1)
        assert rel_l2(got, want) < TOL
