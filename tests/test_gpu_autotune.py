"""The autotuner: it times every plan / launch-shape candidate for a shape,
keeps the fastest in the context's table, the engines then use it, and the
result does not depend on the choice (NRMSE <= 1e-4 vs FP64, and the tuned
and untuned runs agree to 1e-6).  The table round-trips through text."""
import numpy as np
import pytest

from oracle import cs_fp64 as o64
from openkspace_b200 import OksError, _lib
from tests.conftest import crandn, rel_l2

pytestmark = pytest.mark.gpu


def ky_mask(rng, ny, nx, partial=False):
    rows = rng.random(ny) < 0.3
    rows[ny // 2 - 3:ny // 2 + 3] = True
    m = np.zeros((ny, nx), bool)
    if partial:
        m[rows, nx // 4:nx // 4 + nx // 2] = True
    else:
        m[rows, :] = True
    return m


@pytest.mark.parametrize("kind,ny,nx", [(0, 256, 256), (0, 384, 64), (1, 368, 640), (1, 128, 96)])
def test_autotune_choice_applies_and_matches(ctx, rng, kind, ny, nx):
    m = ky_mask(rng, ny, nx, partial=kind == 1)
    k = np.where(m[None], crandn(rng, (4, ny, nx)), 0).astype(np.complex64)
    before = ctx.fista_cs(k, m, 10, 0.02)
    rep = ctx.autotune(kind, ny, nx, nc=4, iters=6)
    try:
        assert rep["kind"] == kind and len(rep["candidates"]) >= 1
        assert rep["chosen"] in [c["params"] for c in rep["candidates"]]
        assert rep["ms"] == min(c["ms"] for c in rep["candidates"])
        table = ctx.autotune_table()
        line = [ln.split() for ln in table.splitlines()]
        assert [kind, ny, 0 if kind == 0 else nx] in [[int(v) for v in ln[:3]] for ln in line]
        after = ctx.fista_cs(k, m, 10, 0.02)
        assert rel_l2(after, before) < 1e-6
        assert rel_l2(after, o64.fista_cs_single_coil(k, m, 10, 0.02)) < 1e-4
        # round trip: clear, load the text back, same table
        ctx.set_option("autotune_clear", 1)
        assert ctx.autotune_table() == ""
        ctx.autotune_load(table)
        assert ctx.autotune_table() == table
    finally:
        ctx.set_option("autotune_clear", 1)


def test_autotune_rejects_bad_input(ctx):
    with pytest.raises(OksError) as e:
        ctx.autotune(2, 64, 64)
    assert e.value.code == _lib.OKS_EINVAL
    with pytest.raises(OksError):
        ctx.autotune(0, 63, 64)
    with pytest.raises(OksError):
        ctx.autotune_load("0 256 0 9 0 1 1 1 2 0\n")
    assert ctx.autotune_table() == ""
