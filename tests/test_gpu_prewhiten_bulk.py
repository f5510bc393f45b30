"""Prewhitening apply (prewhiten.rs:118-142) through the bulk-copy staged
kernel (option prewhiten_bulk = 1; the default -1 takes it for nc <= 8) against the plain-load kernel
(prewhiten_bulk = 0) and the FP64 oracle.  Both kernels share the per-column
arithmetic, so their outputs must be bit-identical; against the oracle the
tolerance is 1e-5 relative L2.  The shapes cover ragged last tiles (ns not a
multiple of the 128-sample tile), one tile, many acquisitions per CTA, the
channel counts of each template bucket, and the cases the launcher hands to
the plain kernel (odd ns, nc above 32, a data pointer off a 16-byte boundary).
"""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from openkspace_b200 import synth
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu


def whitening(rng, nc):
    psi = synth.noise_covariance(nc, 50.0, rng)
    return np.tril(np.linalg.inv(np.linalg.cholesky(psi))).astype(np.complex64)


def apply(ctx, w, data, bulk, offset=0):
    """W s on the device with the given kernel choice; offset > 0 places the
    data that many complex64 elements into a larger buffer."""
    nacq, nc, ns = data.shape
    flat = np.zeros(offset + data.size, np.complex64)
    flat[offset:] = data.ravel()
    d = ctx.to_device(flat)
    dw = ctx.to_device(w)
    ctx.set_option("prewhiten_bulk", bulk)
    try:
        ctx.check(ctx.lib.okscuda_prewhiten_apply(ctx.handle, dw.ptr, d.ptr + 8 * offset, nacq, nc, ns))
    finally:
        ctx.set_option("prewhiten_bulk", -1)
    return d.to_host()[offset:].reshape(data.shape)


@pytest.mark.parametrize("nacq,nc,ns", [(1, 1, 2), (3, 4, 96), (5, 8, 128), (7, 15, 130), (2, 16, 1280),
                                        (40, 15, 256), (3, 32, 640), (4, 9, 1022), (2, 33, 128),
                                        (3, 15, 97)])
def test_bulk_matches_plain_and_oracle(ctx, rng, nacq, nc, ns):
    w = whitening(rng, nc)
    data = crandn(rng, (nacq, nc, ns))
    got = apply(ctx, w, data, 1)
    plain = apply(ctx, w, data, 0)
    assert np.array_equal(got.view(np.uint32), plain.view(np.uint32))
    assert rel_l2(got, o64.prewhiten_apply(w.astype(np.complex128), data)) < 1e-5
    assert ctx.tc_status() == 0


def test_bulk_unaligned_pointer_takes_plain_kernel(ctx, rng):
    """A data pointer 8 bytes off a 16-byte boundary is not eligible for the
    bulk copies; the result is the same."""
    w = whitening(rng, 15)
    data = crandn(rng, (3, 15, 128))
    got = apply(ctx, w, data, 1, offset=1)
    assert rel_l2(got, o64.prewhiten_apply(w.astype(np.complex128), data)) < 1e-5
    assert ctx.tc_status() == 0


def test_bulk_large_batch(ctx, rng):
    """Many tiles per CTA (both stages cycle many times): 600 acquisitions of
    15 channels x 1280 samples, checked against the plain kernel."""
    w = whitening(rng, 15)
    data = crandn(rng, (600, 15, 1280))
    got = apply(ctx, w, data, 1)
    plain = apply(ctx, w, data, 0)
    assert np.array_equal(got.view(np.uint32), plain.view(np.uint32))
    assert ctx.tc_status() == 0
