"""Regenerate the committed golden vectors (tests/golden/cs_golden.npz).

The reference ships no golden outputs for its ``cs`` path and cannot be
built here, so the vectors come from the FP64 oracle (oracle/cs_fp64.py),
whose own pins are the reference's tests restated in
tests/test_oracle_pins.py.  Inputs are seeded (numpy PCG64) and small.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import cs_fp64 as o64  # noqa: E402

# (name, ny, nx, nc, iters, lambda, mask kind, seed)
CASES = [
    ("sq16", 16, 16, 2, 30, 0.02, "rows", 11),
    ("rect24x20", 24, 20, 3, 40, 0.01, "rows", 12),
    ("tall46x16", 46, 16, 2, 25, 0.01, "rows", 13),
    ("sq32_full", 32, 32, 1, 20, 0.05, "full", 14),
    ("sq12_iters0", 12, 12, 2, 0, 0.01, "rows", 15),
    ("rect20x28_2d", 20, 28, 2, 30, 0.02, "random2d", 16),
]


def case_inputs(ny, nx, nc, kind, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    k = (rng.standard_normal((nc, ny, nx)) + 1j * rng.standard_normal((nc, ny, nx))).astype(np.complex64)
    if kind == "rows":
        rows = rng.random(ny) < 0.4
        rows[ny // 2 - 2:ny // 2 + 2] = True
        m = np.repeat(rows[:, None], nx, axis=1)
    elif kind == "full":
        m = np.ones((ny, nx), bool)
    else:
        m = rng.random((ny, nx)) < 0.5
        m[ny // 2 - 2:ny // 2 + 2] = True
    k = np.where(m[None], k, 0).astype(np.complex64)
    return k, m


def main():
    out = {}
    for name, ny, nx, nc, iters, lam, kind, seed in CASES:
        k, m = case_inputs(ny, nx, nc, kind, seed)
        x = o64.fista_cs_single_coil(k, m, iters, lam)
        out[f"{name}__kspace"] = k
        out[f"{name}__mask"] = m.astype(np.uint8)
        out[f"{name}__x"] = x.astype(np.complex128)
        out[f"{name}__rss"] = o64.rss_combine(x)
        out[f"{name}__params"] = np.array([iters, lam])
    np.savez_compressed(os.path.join(HERE, "cs_golden.npz"), **out)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
