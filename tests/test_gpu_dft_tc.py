"""Readout-direction row DFT through the C-ABI: the SIMT mixed-radix FFT and
the tcgen05 tensor-core DFT-as-GEMM (split 3xBF16, FP32 accumulation)
against the FP64 centred transform of cs.rs:141-178 (shift.rs:11-26 shifts).
Tolerances, relative L2: 1e-5 for the FP32 FFT, 3e-5 for the 3xBF16 GEMM
(bf16 hi + lo carries 16 of FP32's 24 mantissa bits per operand)."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu
TOL_SIMT = 1e-5
TOL_TC = 3e-5


def ref_rows(x, inverse, centred):
    a = x.astype(np.complex128)
    if centred:
        a = o64.ifftshift_axis(a, -1)
    a = np.fft.ifft(a, axis=-1) * a.shape[-1] if inverse else np.fft.fft(a, axis=-1)
    if centred:
        a = o64.fftshift_axis(a, -1)
    return a


def test_tc_small_first(ctx, rng):
    """Smallest case first: one 128-row tile, one 256-column tile."""
    x = crandn(rng, (128, 64))
    got = ctx.dft_rows(x, inverse=False, centred=False, engine=1)
    assert ctx.tc_status() == 0
    assert rel_l2(got, ref_rows(x, False, False)) < TOL_TC


@pytest.mark.parametrize("rows,n", [(300, 64), (128, 128), (1000, 320), (736, 368), (515, 640), (40, 30),
                                    (260, 1000), (3, 2048)])
@pytest.mark.parametrize("inverse,centred", [(0, 1), (1, 1), (0, 0)])
def test_engines_match_fp64(ctx, rng, rows, n, inverse, centred):
    x = crandn(rng, (rows, n))
    want = ref_rows(x, inverse, centred)
    simt = ctx.dft_rows(x, inverse=bool(inverse), centred=bool(centred), engine=0)
    tc = ctx.dft_rows(x, inverse=bool(inverse), centred=bool(centred), engine=1)
    assert ctx.tc_status() == 0
    assert rel_l2(simt, want) < TOL_SIMT
    assert rel_l2(tc, want) < TOL_TC


def test_tc_in_place_and_errors(ctx, rng):
    from openkspace_b200 import OksError, _lib
    x = crandn(rng, (200, 320))
    got = ctx.dft_rows(x, inverse=True, centred=True, engine=1, in_place=True)
    assert ctx.tc_status() == 0
    assert rel_l2(got, ref_rows(x, 1, 1)) < TOL_TC
    with pytest.raises(OksError) as e:
        ctx.dft_rows(crandn(rng, (2, 4096)), engine=1)
    assert e.value.code == _lib.OKS_ENOTSUP
    d = ctx.to_device(x)
    assert ctx.lib.okscuda_dft_rows(ctx.handle, d.ptr, d.ptr, 200, 320, 0, 1, 7) == _lib.OKS_EINVAL
    assert ctx.lib.okscuda_dft_rows(ctx.handle, d.ptr, d.ptr, 0, 320, 0, 1, 1) == 0


def partial_row_mask(rng, ny, nx, frac=0.35):
    rows = rng.random(ny) < frac
    rows[ny // 2 - 2:ny // 2 + 2] = True
    m = np.zeros((ny, nx), bool)
    m[rows, nx // 4:nx // 4 + nx // 2] = True
    return m


@pytest.mark.parametrize("ny,nx,iters", [(368, 640, 12), (64, 96, 20), (256, 256, 10)])
def test_fista_row_engine_tensor_cores(ctx, rng, ny, nx, iters):
    """The 2-D-mask engine with its readout transforms on the tensor cores
    (row_engine 1) against FP64 and against the SIMT engine: NRMSE <= 1e-4."""
    m = partial_row_mask(rng, ny, nx)
    k = np.where(m[None], crandn(rng, (3, ny, nx)), 0).astype(np.complex64)
    want = o64.fista_cs_single_coil(k, m, iters, 0.02)
    simt = ctx.fista_cs(k, m, iters, 0.02)
    ctx.set_option("row_engine", 1)
    try:
        tc = ctx.fista_cs(k, m, iters, 0.02)
    finally:
        ctx.set_option("row_engine", 0)
    assert ctx.tc_status() == 0
    assert o64.nrmse(tc, want) < 1e-4
    assert o64.nrmse(simt, want) < 1e-4
    assert o64.nrmse(tc, simt) < 1e-4


def test_fista_row_engine_tc_ragged_and_per_slice_masks(ctx, rng):
    """Different masks per slice (non-contiguous union of sampled columns)
    through the volume path with the tensor-core row pass."""
    nc, nz, ny, nx = 2, 3, 32, 48
    ms = []
    for _ in range(nz):
        mm = np.zeros((ny, nx), bool)
        rows = rng.random(ny) < 0.4
        rows[ny // 2] = True
        cols = rng.random(nx) < 0.6
        mm[np.ix_(rows, cols)] = True
        ms.append(mm)
    m = np.stack(ms)
    k = np.where(m[None], crandn(rng, (nc, nz, ny, nx)), 0).astype(np.complex64)
    ctx.set_option("row_engine", 1)
    try:
        rss = ctx.cs_volume(k, m, 15, 0.02)
    finally:
        ctx.set_option("row_engine", 0)
    assert ctx.tc_status() == 0
    want = o64.csrss_from_kspace(k, m, 15, 0.02)
    assert o64.nrmse(rss, want) < 1e-4


def test_bounded_wait_times_out_and_returns(ctx, rng):
    """The tensor-core kernel's bounded waits: with the gate test on, every
    CTA first waits on a device word that nothing sets, for at most ~1 ms of
    clock cycles; the call returns, okscuda_tc_status reports the time-out
    (code 7) and clears it, and the next launch (gate off) is correct -- the
    context stays usable."""
    x = crandn(rng, (256, 128))
    ctx.set_option("tc_gate_test", 2_000_000)
    try:
        ctx.dft_rows(x, inverse=False, centred=True, engine=1)
        ctx.synchronize()
        assert ctx.tc_status() == 7
        assert ctx.tc_status() == 0          # read and cleared
    finally:
        ctx.set_option("tc_gate_test", 0)
    got = ctx.dft_rows(x, inverse=False, centred=True, engine=1)
    assert ctx.tc_status() == 0
    assert rel_l2(got, ref_rows(x, False, True)) < TOL_TC
