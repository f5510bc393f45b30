"""Parity of the arbitrary-2-D-mask FISTA engine (masks not constant along kx,
e.g. the partial rows the reference's reader produces after readout
oversampling removal, reader.rs:394-457) against the oracle.  Tolerance:
relative L2 <= 1e-4 vs the FP32 restatement and NRMSE <= 1e-4 vs FP64."""
import os

import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import csref
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu
TOL_CS = 1e-4
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cs_golden.npz")


def partial_row_mask(rng, ny, nx, frac=0.35):
    """ky rows sampled only over the central half of kx (the placement of a
    readout shortened 2x by oversampling removal)."""
    rows = rng.random(ny) < frac
    rows[ny // 2 - 2:ny // 2 + 2] = True
    m = np.zeros((ny, nx), bool)
    m[rows, nx // 4:nx // 4 + nx // 2] = True
    return m


@pytest.mark.parametrize("ny,nx,iters", [(16, 16, 20), (24, 40, 25), (46, 20, 15), (64, 128, 10),
                                         (368, 64, 8), (48, 640, 6), (2, 4, 5)])
def test_partial_row_masks(ctx, rng, ny, nx, iters):
    m = partial_row_mask(rng, ny, nx)
    k = np.where(m[None], crandn(rng, (2, ny, nx)), 0).astype(np.complex64)
    got = ctx.fista_cs(k, m, iters, 0.03)
    assert rel_l2(got, o64.fista_cs_single_coil(k, m, iters, 0.03)) < TOL_CS
    want32 = np.stack([csref.fista_cs_single_coil(k[c], m, iters, 0.03) for c in range(2)])
    assert rel_l2(got, want32) < TOL_CS


@pytest.mark.parametrize("ny,nx,iters", [(368, 640, 6), (256, 256, 10), (320, 384, 5), (384, 320, 5),
                                         (192, 512, 4), (512, 192, 4)])
def test_register_passes_match_generic_and_oracle(ctx, rng, ny, nx, iters):
    """Register-resident column/row passes (compile-time plans) against the
    generic shared-memory passes and FP64, including the reference's
    368 x 640 partial-row grid of the oversampled workload."""
    m = partial_row_mask(rng, ny, nx)
    k = np.where(m[None], crandn(rng, (2, ny, nx)), 0).astype(np.complex64)
    got = ctx.fista_cs(k, m, iters, 0.02)
    ctx.set_option("col_engine", 1)
    try:
        gen = ctx.fista_cs(k, m, iters, 0.02)
    finally:
        ctx.set_option("col_engine", 0)
    assert rel_l2(got, gen) < 1e-5
    assert rel_l2(got, o64.fista_cs_single_coil(k, m, iters, 0.02)) < TOL_CS


@pytest.mark.parametrize("ny,nx", [(20, 28), (32, 32), (10, 6)])
def test_random_2d_masks(ctx, rng, ny, nx):
    m = rng.random((ny, nx)) < 0.45
    k = np.where(m[None], crandn(rng, (3, ny, nx)), 0).astype(np.complex64)
    got = ctx.fista_cs(k, m, 20, 0.02)
    assert rel_l2(got, o64.fista_cs_single_coil(k, m, 20, 0.02)) < TOL_CS


def test_golden_2d_mask(ctx):
    g = np.load(GOLDEN)
    name = "rect20x28_2d"
    k, m = g[f"{name}__kspace"], g[f"{name}__mask"].astype(bool)
    iters, lam = g[f"{name}__params"]
    assert not np.all(m == m[:, :1])
    got = ctx.fista_cs(k, m, int(iters), float(lam))
    assert rel_l2(got, g[f"{name}__x"]) < TOL_CS


def test_2d_iters0_and_empty(ctx, rng):
    ny, nx = 12, 16
    m = partial_row_mask(rng, ny, nx)
    k = np.where(m, crandn(rng, (ny, nx)), 0).astype(np.complex64)
    assert rel_l2(ctx.fista_cs(k, m, 0, 0.01), o64.centred_ifft2(k)) < 1e-5
    m0 = np.zeros((ny, nx), bool)
    m0[3, 2] = True   # not constant along kx, one sample
    z = ctx.fista_cs(k, m0, 4, 0.01)
    assert rel_l2(z, o64.fista_cs_single_coil(k, m0, 4, 0.01)) < TOL_CS


def test_volume_with_partial_rows_matches_oracle(ctx, rng):
    """strategy.rs:849-885 with per-slice partial-row masks."""
    nc, nz, ny, nx = 2, 3, 24, 32
    m = np.stack([partial_row_mask(rng, ny, nx) for _ in range(nz)])
    k = np.where(m[None], crandn(rng, (nc, nz, ny, nx)), 0).astype(np.complex64)
    rss = ctx.cs_volume(k, m, 12, 0.02, crop=(24, 16))
    want = o64.maybe_crop(o64.csrss_from_kspace(k, m, 12, 0.02), (16, 24, 1))
    assert o64.nrmse(rss, want) < TOL_CS


def ragged_row_mask(rng, ny, nx, frac=0.35):
    """Sampled rows with windows of different extent per row: not
    separable, so the column pass reads the byte mask."""
    rows = np.flatnonzero(rng.random(ny) < frac)
    m = np.zeros((ny, nx), bool)
    for r in rows:
        lo = int(rng.integers(0, nx // 4)) * 2
        m[r, lo:nx - int(rng.integers(0, nx // 4)) * 2] = True
    m[ny // 2, :] = True
    return m


@pytest.mark.parametrize("ny,nx,iters", [(368, 640, 5), (256, 256, 6), (384, 320, 4)])
def test_mask_forms_and_launch_forms_agree(ctx, rng, ny, nx, iters):
    """Separable masks read as row/column bits vs as bytes, the two register
    budgets of the 2-D passes, persistent vs one-CTA-per-unit grids, one vs
    two chunks in flight and the pipelined vs plain column pass give the
    same result; a ragged (non-separable)
    mask takes the byte path and matches FP64."""
    m = partial_row_mask(rng, ny, nx)
    k = np.where(m[None], crandn(rng, (5, ny, nx)), 0).astype(np.complex64)
    want = o64.fista_cs_single_coil(k, m, iters, 0.02)
    forms = [dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2),
             dict(mask_bits=0, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2),
             dict(mask_bits=1, occ2d=0, persist2d=0, fista2d_streams=1, fista2d_chunk=2),
             dict(mask_bits=1, occ2d=1, persist2d=0, fista2d_streams=3, fista2d_chunk=1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=0),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=3),
             dict(mask_bits=1, occ2d=2, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=1),
             dict(mask_bits=1, occ2d=2, persist2d=1, fista2d_streams=1, fista2d_chunk=2, prefetch2d=3),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=5),
             dict(mask_bits=1, occ2d=1, persist2d=0, fista2d_streams=1, fista2d_chunk=3, prefetch2d=4),
             dict(mask_bits=0, occ2d=2, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=5),
             dict(mask_bits=1, occ2d=3, persist2d=1, fista2d_streams=2, fista2d_chunk=2, prefetch2d=1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=5),
             dict(mask_bits=0, occ2d=1, persist2d=1, fista2d_streams=1, fista2d_chunk=3, col2d_lanes=6),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=7),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=3, col2d_lanes=8),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=4),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=-1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=9),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=3, col2d_lanes=10),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=1, fista2d_chunk=2, col2d_lanes=11),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=12),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, row2d_ctas=1, col2d_ctas=1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=3, row2d_ctas=2, col2d_ctas=2),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, pdl2d=1),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=2, col2d_lanes=14),
             dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=1, fista2d_chunk=3, pdl2d=1, col2d_lanes=-1)]
    default = dict(mask_bits=1, occ2d=1, persist2d=1, fista2d_streams=2, fista2d_chunk=0, prefetch2d=1, col2d_lanes=0,
                   row2d_ctas=0, col2d_ctas=0, pdl2d=0)
    results = []
    try:
        for form in forms:
            for name, v in form.items():
                ctx.set_option(name, v)
            results.append(ctx.fista_cs(k, m, iters, 0.02))
    finally:
        for name, v in default.items():
            ctx.set_option(name, v)
    for r in results:
        assert rel_l2(r, results[0]) < 1e-6
        assert rel_l2(r, want) < TOL_CS
    assert ctx.tc_status() == 0                  # no bounded wait of the bulk-copy row pass ran out
    mr = ragged_row_mask(rng, ny, nx)
    kr = np.where(mr[None], crandn(rng, (2, ny, nx)), 0).astype(np.complex64)
    assert rel_l2(ctx.fista_cs(kr, mr, iters, 0.02), o64.fista_cs_single_coil(kr, mr, iters, 0.02)) < TOL_CS


def row_set_mask(ny, nx, rows):
    """Separable mask: the given ky rows over the central half of kx."""
    m = np.zeros((ny, nx), bool)
    m[np.asarray(rows, int), nx // 4:nx // 4 + nx // 2] = True
    return m


@pytest.mark.parametrize("rows", ["r4_centre", "r4_offset", "r3", "random20", "one_row", "all", "class_edge"])
@pytest.mark.parametrize("form", [9, 10, 11, 12, 13, 14])
def test_pruned_368_column_pass(ctx, rng, rows, form):
    """The 368 column pass pruned to the sampled rows (col2d_lanes 9-14)
    against the full register pass and FP64, for row sets that exercise
    every pruning case: R = 4 plus a centre block (the precision workload's
    pattern, dense class and sparse classes), R = 4 shifted by one row, R = 3
    (every class partly sampled), random rows, a single row (one need bit),
    every row (nothing pruned), and rows at the ends of the 92-row blocks."""
    ny, nx, iters = 368, 96, 6
    rset = {"r4_centre": list(range(0, ny, 4)) + list(range(ny // 2 - 15, ny // 2 + 15)),
            "r4_offset": list(range(1, ny, 4)) + [ny // 2],
            "r3": list(range(2, ny, 3)),
            "random20": list(np.flatnonzero(rng.random(ny) < 0.2)) + [ny // 2],
            "one_row": [ny // 2 + 5],
            "all": list(range(ny)),
            "class_edge": [0, 91, 92, 183, 276, 367, 3, 95]}[rows]
    m = row_set_mask(ny, nx, sorted(set(rset)))
    k = np.where(m[None], crandn(rng, (3, ny, nx)), 0).astype(np.complex64)
    ctx.set_option("col2d_lanes", -1)
    base = ctx.fista_cs(k, m, iters, 0.02)
    ctx.set_option("col2d_lanes", form)
    try:
        got = ctx.fista_cs(k, m, iters, 0.02)
    finally:
        ctx.set_option("col2d_lanes", 0)
    assert rel_l2(got, base) < 1e-5
    assert rel_l2(got, o64.fista_cs_single_coil(k, m, iters, 0.02)) < TOL_CS


def test_pruned_368_column_pass_full_width(ctx, rng):
    """The precision workload's grid (368 x 640, R = 4 plus 8 % centre over
    the central half of kx) through the pruned form (the default at ny = 368)
    against the column-pair pass, with the CUDA graph
    (second call of a shape) and two chunks in flight, for two row offsets."""
    ny, nx, iters = 368, 640, 5
    for off in (0, 2):
        rows = sorted(set(range(off, ny, 4)) | set(range(ny // 2 - 15, ny // 2 + 15)))
        m = row_set_mask(ny, nx, rows)
        k = np.where(m[None], crandn(rng, (5, ny, nx)), 0).astype(np.complex64)
        ctx.set_option("col2d_lanes", -1)
        base = ctx.fista_cs(k, m, iters, 0.02)
        ctx.set_option("col2d_lanes", 0)
        try:
            got = [ctx.fista_cs(k, m, iters, 0.02) for _ in range(3)]   # direct, captured, replayed
        finally:
            ctx.set_option("col2d_lanes", 0)
        for g in got:
            assert rel_l2(g, base) < 1e-5
        assert rel_l2(got[-1], o64.fista_cs_single_coil(k, m, iters, 0.02)) < TOL_CS


def test_graph_replay_matches_direct_launches(ctx, rng):
    """The CUDA-graph form of the 2-D engine: the first call of a shape runs
    the launches directly, the second captures and replays them, later calls
    replay; every call sees its own k-space and masks (new data each call,
    in place and out of place) and matches the direct launches and FP64."""
    ny, nx, iters = 368, 640, 4
    results = []
    try:
        for graph in (0, 1):
            ctx.set_option("graph2d", graph)
            r = np.random.default_rng(99)
            out = []
            for call in range(4):
                m = partial_row_mask(r, ny, nx)
                k = np.where(m[None], crandn(r, (13, ny, nx)), 0).astype(np.complex64)
                out.append((ctx.fista_cs(k, m, iters, 0.02), k, m))
            results.append(out)
    finally:
        ctx.set_option("graph2d", 1)
    for (g0, k, m), (g1, _, _) in zip(results[0], results[1]):
        assert rel_l2(g1, g0) < 1e-6
    g_last, k, m = results[1][-1]
    assert o64.nrmse(g_last[:2], o64.fista_cs_single_coil(k[:2], m, iters, 0.02)) < TOL_CS
    # in place (output buffer = input buffer), replayed
    d = ctx.to_device(k)
    ctx.fista_cs(d, m, iters, 0.02, out=d)
    assert rel_l2(d.to_host(), g_last) < 1e-6
