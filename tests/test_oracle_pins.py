"""Pins of the oracle: every known-answer and property test the reference
holds for the ``cs`` path, restated against both restatements (FP64 numpy
``cs_fp64`` and FP32 C ``csref``).  Reference test locations are relative to
crates/openkspace-recon/src/."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from oracle import csref
from tests.conftest import crandn, rel_l2


# ---------------------------------------------------------------- cs.rs tests
def _ramp8():
    i, j = np.meshgrid(np.arange(8), np.arange(8), indexing="ij")
    return ((i + j) + 1j * (i - j) * 0.3).astype(np.complex64)


@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_fft_pair_is_unitary(impl):
    """cs.rs:224-256: energy within 1e-3, round trip within 1e-4 per element."""
    x = _ramp8()
    fwd = o64.centred_fft2 if impl == "fp64" else (lambda a: csref.centred_fft2(a))
    inv = o64.centred_ifft2 if impl == "fp64" else (lambda a: csref.centred_fft2(a, True))
    y = fwd(x)
    e_in = np.sum(np.abs(x) ** 2)
    assert abs(e_in - np.sum(np.abs(y) ** 2)) < 1e-3
    z = inv(y)
    assert np.max(np.abs(z - x)) < 1e-4


def sparse_phantom_case():
    """cs.rs:258-295 inputs: 16x16, four deltas, R=2 + 4 centre ky lines."""
    ny = nx = 16
    truth = np.zeros((ny, nx), np.complex64)
    truth[5, 4] = 1.0
    truth[10, 11] = 0.8
    truth[3, 12] = 0.6
    truth[12, 3] = 0.5
    k = o64.centred_fft2(truth)
    mask = np.zeros((ny, nx), bool)
    for i in range(ny):
        if i % 2 == 0 or (ny // 2 - 2 <= i < ny // 2 + 2):
            mask[i, :] = True
    kzf = np.where(mask, k, 0).astype(np.complex64)
    return truth, kzf, mask


@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_cs_recovers_sparse_phantom(impl):
    """cs.rs:258-321: 200 iterations at lambda 0.02, cs_err < 0.8 zf_err."""
    truth, kzf, mask = sparse_phantom_case()
    zf = o64.centred_ifft2(kzf)
    zf_err = np.linalg.norm((zf - truth).ravel())
    f = o64.fista_cs_single_coil if impl == "fp64" else csref.fista_cs_single_coil
    rec = f(kzf, mask, 200, 0.02)
    cs_err = np.linalg.norm((rec - truth).ravel())
    assert cs_err < 0.8 * zf_err


def test_cs_shape_and_odd_errors():
    """cs.rs:66-74: mask shape mismatch and odd dimensions are errors."""
    k = np.zeros((8, 8), np.complex64)
    with pytest.raises(ValueError):
        o64.fista_cs_single_coil(k, np.ones((8, 6), bool), 1, 0.01)
    with pytest.raises(ValueError):
        o64.fista_cs_single_coil(np.zeros((7, 8), np.complex64), np.ones((7, 8), bool), 1, 0.01)
    with pytest.raises(ValueError):
        csref.fista_cs_single_coil(np.zeros((6, 5), np.complex64), np.ones((6, 5), bool), 1, 0.01)


# ----------------------------------------------------------- wavelet.rs tests
@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_haar_roundtrip_recovers_input(impl):
    """wavelet.rs:105-121."""
    i, j = np.meshgrid(np.arange(8), np.arange(8), indexing="ij")
    x = (i + 1j * j * 0.3).astype(np.complex64)
    fw = o64.haar_forward if impl == "fp64" else csref.haar_forward
    iv = o64.haar_inverse if impl == "fp64" else csref.haar_inverse
    assert np.max(np.abs(iv(fw(x)) - x)) < 1e-5


@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_haar_preserves_energy(impl):
    """wavelet.rs:123-133."""
    x = np.zeros((4, 4), np.complex64)
    x[0, 0] = 1.0
    x[1, 2] = 1j
    x[3, 3] = 0.5 - 0.5j
    fw = o64.haar_forward if impl == "fp64" else csref.haar_forward
    assert abs(np.sum(np.abs(x) ** 2) - np.sum(np.abs(fw(x)) ** 2)) < 1e-5


def test_soft_threshold_semantics():
    """wavelet.rs:80-99: LL untouched, |z| <= lambda -> 0, else shrink."""
    y = np.full((4, 4), 0.375 + 0.5j, np.complex64)   # |z| = 0.625 exactly
    y[3, 3] = 0.1
    for f in (o64.soft_threshold_details, csref.soft_threshold_details):
        r = f(y, 0.25)
        assert np.allclose(r[:2, :2], y[:2, :2])
        assert np.allclose(r[0, 2], (0.375 + 0.5j) * 0.6, atol=1e-6)
        assert r[3, 3] == 0
        assert np.all(f(y, 0.625)[2:, :] == 0)   # m <= lambda with equality -> 0


# ------------------------------------------------------------- shift.rs tests
def test_shift_semantics():
    """shift.rs:62-84."""
    a = np.arange(4).astype(np.complex64)
    assert np.array_equal(o64.fftshift_axis(a, 0).real, [2, 3, 0, 1])
    b = np.arange(5).astype(np.complex64)
    assert np.array_equal(o64.fftshift_axis(b, 0).real, [2, 3, 4, 0, 1])
    assert np.array_equal(o64.ifftshift_axis(o64.fftshift_axis(b, 0), 0), b)


# --------------------------------------------------------------- fft.rs tests
def test_ifft2_impulse_gives_constant():
    """fft.rs:91-112."""
    n = 8
    k = np.zeros((n, n), np.complex64)
    k[n // 2, n // 2] = 1.0
    r = o64.ifft2_inplace(k, (0, 1))
    assert np.max(np.abs(np.abs(r) - 1.0 / (n * n))) < 1e-6


def test_ifft2_parseval():
    """fft.rs:114-135."""
    n = 16
    k = np.zeros((n, n), np.complex64)
    k[0, 0] = 1.0
    k[1, 2] = 0.5 - 0.25j
    before = np.sum(np.abs(k) ** 2)
    after = np.sum(np.abs(o64.ifft2_inplace(k, (0, 1))) ** 2)
    assert abs(after - before / (n * n)) < 1e-5


def test_ifft1_decouples_from_2d():
    """fft.rs:160-192: ifft3 == ifft2_axes23(ifft1_axis1(k)) (and the FP32
    restatement's kz IFFT agrees)."""
    nz, ny, nx = 4, 6, 6
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    k = ((z + 1.0) * 0.5 * ((y - 2.0) + 1j * x * 0.25)).astype(np.complex64)
    a = o64.ifft2_inplace(o64.ifft1_inplace(k, 0), (1, 2))
    full = o64.ifftshift_axis(o64.ifftshift_axis(o64.ifftshift_axis(k, 0), 1), 2)
    full = np.fft.ifftn(full)
    full = o64.fftshift_axis(o64.fftshift_axis(o64.fftshift_axis(full, 0), 1), 2)
    assert np.max(np.abs(a - full)) < 1e-4
    b = csref.ifft1_axis(k, 0)
    assert np.max(np.abs(b - o64.ifft1_inplace(k, 0))) < 1e-5


@pytest.mark.parametrize("n", [5, 7, 192])
def test_ifft1_odd_and_kz_lengths(n, rng):
    k = crandn(rng, (3, n, 4))
    assert rel_l2(csref.ifft1_axis(k, 1), o64.ifft1_inplace(k, 1)) < 1e-6


# -------------------------------------------------------- prewhiten.rs tests
def lcg_whitening_fixture():
    """prewhiten.rs:225-266: nc = 4, ns = 4096, deterministic LCG noise through
    a known lower-triangular L."""
    nc, ns = 4, 4096
    l_true = np.zeros((nc, nc), np.complex64)
    for i in range(nc):
        l_true[i, i] = 1.0 + 0.5 * i
        for j in range(i):
            l_true[i, j] = 0.1 * (i + j) - 0.05j * i
    state = 0xDEADBEEFCAFEF00D
    mask64 = (1 << 64) - 1
    vals = np.empty(2 * nc * ns, np.float32)
    for q in range(vals.size):
        state = (state * 6364136223846793005 + 1442695040888963407) & mask64
        u = np.float32((state >> 33) & 0xFFFFFFFF) / np.float32(4294967295.0)
        vals[q] = np.float32(u - np.float32(0.5))
    n0 = (vals[0::2] + 1j * vals[1::2]).astype(np.complex64).reshape(ns, nc)
    data = np.zeros((nc, ns), np.complex64)
    for i in range(nc):
        data[i] = np.sum(l_true[i, :i + 1][None, :] * n0[:, :i + 1], axis=1)
    return data


@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_whitens_correlated_noise_to_identity(impl):
    """prewhiten.rs:218-302: whitened covariance within 0.08 of I."""
    data = lcg_whitening_fixture()
    if impl == "fp64":
        w = o64.prewhitener_from_noise([data])
        out = o64.prewhiten_apply(w, data)
    else:
        w = csref.prewhiten_fit(data)
        out = csref.prewhiten_apply(w, data)
    assert w is not None
    nc, ns = data.shape
    cov = out @ np.conj(out.T) / (ns - 1)
    assert np.max(np.abs(cov.real - np.eye(nc))) < 0.08
    assert np.max(np.abs(cov.imag)) < 0.08


def test_prewhiten_skips():
    """prewhiten.rs:49-66, 161-164: no scans / too few samples / not PD -> None."""
    assert o64.prewhitener_from_noise([]) is None
    assert o64.prewhitener_from_noise([np.ones((4, 3), np.complex64)]) is None
    assert csref.prewhiten_fit(np.ones((4, 3), np.complex64)) is None
    rank1 = np.ones((3, 10), np.complex64)   # Psi singular -> Cholesky fails
    assert o64.prewhitener_from_noise([rank1]) is None
    assert csref.prewhiten_fit(rank1) is None


def test_prewhiten_fp32_matches_fp64(rng):
    data = crandn(rng, (15, 256))
    w64 = o64.prewhitener_from_noise([data])
    w32 = csref.prewhiten_fit(data)
    assert rel_l2(w32, w64) < 1e-5


# ------------------------------------------------------ oversampling.rs tests
def test_oversampling_constructor_rules():
    """oversampling.rs:216-234."""
    assert o64.oversampling_ratio(256, 256) is None
    assert o64.oversampling_ratio(256, 512) is None
    assert o64.oversampling_ratio(256, 0) is None
    assert o64.oversampling_ratio(300, 256) is None
    assert o64.oversampling_ratio(512, 256) == 2
    assert o64.oversampling_ratio(4608, 512) is None   # ratio 9 > 8


@pytest.mark.parametrize("impl", ["fp64", "fp32"])
def test_oversampling_preserves_dc_only_signal(impl):
    """oversampling.rs:236-275: DC spike scaled by M/N at the new centre."""
    enc, rec = 16, 8
    d = np.zeros((1, enc), np.complex64)
    d[0, enc // 2] = 10.0
    out = (o64.oversampling_apply(d, enc, rec) if impl == "fp64" else csref.oversampling_apply(d, enc, rec))[0]
    for i in range(rec):
        want = 10.0 * rec / enc if i == rec // 2 else 0.0
        assert abs(out[i] - want) < 1e-4


def test_oversampling_passes_mismatched_through():
    """oversampling.rs:277-293."""
    d = np.full((2, 64), 1 + 2j, np.complex64)
    assert np.array_equal(o64.oversampling_apply(d, 512, 256), d)


def test_oversampling_fp32_matches_fp64(rng):
    d = crandn(rng, (3, 15, 640))
    assert rel_l2(csref.oversampling_apply(d, 640, 320), o64.oversampling_apply(d, 640, 320)) < 1e-6


# ------------------------------------------------------- coil.rs / crop.rs
def test_rss_known_answers():
    """coil.rs:34-53: sqrt(50) and 13."""
    a = np.array([3, 4, 5], np.complex64).reshape(3, 1, 1)
    assert abs(o64.rss_combine(a)[0, 0] - np.sqrt(50.0)) < 1e-6
    b = np.array([3 + 4j, 12j], np.complex64).reshape(2, 1, 1)
    assert abs(o64.rss_combine(b)[0, 0] - 13.0) < 1e-6


def test_crop_centering():
    """crop.rs:33-53."""
    v = np.zeros((1, 4, 8), np.float32)
    v[0, 1:3, 2:6] = 1.0
    c = o64.center_crop_3d(v, (1, 2, 4))
    assert c.shape == (1, 2, 4) and np.all(c == 1.0)
    assert o64.center_crop_3d(np.ones((2, 3, 5)), (10, 10, 10)).shape == (2, 3, 5)
    # strategy.rs:227-253: z is cropped only when recon z >= 2
    assert o64.maybe_crop(np.ones((3, 8, 8)), (4, 6, 1)).shape == (3, 6, 4)


# --------------------------------------------- restatements agree with each other
@pytest.mark.parametrize("ny,nx", [(16, 16), (24, 20), (32, 48), (46, 16)])
def test_fista_fp32_restatement_matches_fp64(ny, nx, rng):
    k = crandn(rng, (ny, nx))
    m = np.zeros((ny, nx), bool)
    m[rng.random(ny) < 0.4] = True
    m[ny // 2 - 2:ny // 2 + 2] = True
    a = csref.fista_cs_single_coil(k, m, 40, 0.05)
    b = o64.fista_cs_single_coil(k, m, 40, 0.05)
    assert rel_l2(a, b) < 1e-5


def test_csrss_threads_agree(rng):
    k = crandn(rng, (3, 2, 16, 12))
    m = np.zeros((2, 16, 12), bool)
    m[:, ::2] = True
    r1 = csref.csrss(k, m, 20, 0.01, nthreads=1)
    r4 = csref.csrss(k, m, 20, 0.01, nthreads=4)
    assert np.array_equal(r1, r4)
    r64 = o64.csrss_from_kspace(k, m, 20, 0.01)
    assert rel_l2(r1, r64) < 1e-5


# ------------------------------------------------------------ phasecorr.rs
def test_phasecorr_empty_corrector_is_noop():
    """phasecorr.rs:189-196: no navigators, the line is unchanged."""
    corr = o64.phase_corrector_from_acqs([])
    assert corr == {}
    d = np.array([[1.0 + 2.0j]])
    assert np.array_equal(o64.phase_correct_apply(corr, d, 0, 0), d)


def test_phasecorr_removes_constant_phase_offset():
    """phasecorr.rs:198-228: a navigator at a constant phase pi/3 makes an
    image line carrying the same phase on a real ramp real again."""
    ns, phi = 8, np.pi / 3
    nav = np.full((1, ns), np.exp(1j * phi))
    corr = o64.phase_corrector_from_acqs([(0, 0, nav)])
    assert set(corr) == {(0, 0)}
    img = (np.exp(1j * phi) * np.arange(1, ns + 1))[None]
    got = o64.phase_correct_apply(corr, img, 0, 0)
    assert np.all(np.abs(got.real - np.arange(1, ns + 1)) < 1e-4) and np.all(np.abs(got.imag) < 1e-4)


def test_phasecorr_binning_rules():
    """phasecorr.rs:70-103, 141-168: coil sums averaged per (slice, segment);
    a scan with another ns is dropped; empty scans are skipped; a line takes
    its (slice, segment) bin, else (65535, segment), else stays as it is; only
    the first min(ns, len(c)) samples are corrected; |avg| < 1e-20 gives 1."""
    rng = np.random.default_rng(3)
    a = rng.standard_normal((2, 6)) + 1j * rng.standard_normal((2, 6))
    b = rng.standard_normal((3, 6)) + 1j * rng.standard_normal((3, 6))
    odd = rng.standard_normal((2, 5)) + 1j * rng.standard_normal((2, 5))
    fall = rng.standard_normal((1, 4)) + 1j * rng.standard_normal((1, 4))
    zero = np.zeros((1, 6), complex)
    corr = o64.phase_corrector_from_acqs([(0, 1, a), (0, 1, odd), (0, 1, b), (0, 2, np.zeros((0, 6))),
                                          (65535, 3, fall), (1, 1, zero)])
    avg = (a.sum(0) + b.sum(0)) / 2
    assert np.allclose(corr[(0, 1)], np.conj(avg) / np.abs(avg))
    assert (0, 2) not in corr
    assert np.array_equal(corr[(1, 1)], np.ones(6, complex))
    line = rng.standard_normal((2, 6)) + 1j * rng.standard_normal((2, 6))
    assert np.allclose(o64.phase_correct_apply(corr, line, 0, 1), line * corr[(0, 1)])
    got = o64.phase_correct_apply(corr, line, 5, 3)          # slice 5 has no bin: the (65535, 3) one
    assert np.allclose(got[:, :4], line[:, :4] * corr[(65535, 3)]) and np.array_equal(got[:, 4:], line[:, 4:])
    assert np.array_equal(o64.phase_correct_apply(corr, line, 0, 7), line)


# ----------------------------------------------------------------- sense.rs
def _sense_r2_case():
    """sense.rs:262-341: 4 Gaussian coils at the corners, a rectangle with a
    dot, every other ky line kept (plain FFT along y)."""
    nc, ny, nx, r = 4, 32, 24, 2
    truth = np.zeros((ny, nx), np.float32)
    truth[6:26, 4:20] = 1.0
    truth[14:18, 10:14] = 0.3
    maps = np.zeros((nc, ny, nx), np.complex64)
    yy, xx = np.meshgrid(np.arange(ny, dtype=np.float32), np.arange(nx, dtype=np.float32), indexing="ij")
    for c, (fy, fx) in enumerate([(0.25, 0.25), (0.25, 0.75), (0.75, 0.25), (0.75, 0.75)]):
        mag = np.exp(-((yy - fy * ny) ** 2 + (xx - fx * nx) ** 2) / 200.0)
        maps[c] = mag * np.exp(1j * 0.2 * c)
    k = np.fft.fft(maps * truth, axis=1)
    k[:, np.arange(ny) % r != 0, :] = 0
    aliased = np.fft.ifft(k, axis=1).astype(np.complex64)
    return truth, maps, aliased, r


def test_sense_unfold_r2_phantom_both_oracles():
    from oracle import sense_fp64 as sref
    truth, maps, aliased, r = _sense_r2_case()
    assert np.sqrt(np.sum(np.abs(aliased[:, 0] - aliased[:, 32 // r]) ** 2)) < 1e-3
    for out in (sref.sense_unfold_1d(aliased, maps, r, 1e-5)[0], csref.sense_unfold(aliased, maps, r, 1e-5)[0]):
        m = np.abs(out)
        assert np.sqrt(np.sum((truth - m) ** 2) / np.sum(truth ** 2)) < 0.1


def test_sense_r1_passthrough_and_unit_gfactor():
    from oracle import sense_fp64 as sref
    nc, ny, nx = 2, 8, 6                                 # sense.rs:353-393
    maps = np.ones((nc, ny, nx), np.complex64)
    y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    aliased = np.stack([np.sin(y * 0.1 + x * 0.05 + c) for c in range(nc)]).astype(np.complex64)
    for out in (sref.sense_unfold_1d(aliased, maps, 1, 0.0)[0], csref.sense_unfold(aliased, maps, 1, 0.0)[0]):
        assert np.abs(out - aliased.mean(0)).max() < 1e-4
    maps3 = np.ones((3, 6, 5), np.complex64)              # sense.rs:398-421: g = 1 with R = 1
    for g in (sref.sense_unfold_1d(np.zeros_like(maps3), maps3, 1, 0.0, gfactor=True)[1],
              csref.sense_unfold(np.zeros_like(maps3), maps3, 1, 0.0, gfactor=True)[1]):
        assert np.abs(g - 1.0).max() < 1e-5


def test_sense_fp32_restatement_matches_fp64():
    from oracle import sense_fp64 as sref
    rng = np.random.default_rng(8)
    nc, ny, nx, r = 6, 24, 10, 3
    maps = (rng.standard_normal((nc, ny, nx)) + 1j * rng.standard_normal((nc, ny, nx))).astype(np.complex64)
    al = (rng.standard_normal((nc, ny, nx)) + 1j * rng.standard_normal((nc, ny, nx))).astype(np.complex64)
    o32, g32 = csref.sense_unfold(al, maps, r, 1e-3, gfactor=True)
    o64, g64 = sref.sense_unfold_1d(al, maps, r, 1e-3, gfactor=True)
    assert np.linalg.norm(o32 - o64) / np.linalg.norm(o64) < 1e-5
    assert np.linalg.norm(g32 - g64) / np.linalg.norm(g64) < 1e-5
