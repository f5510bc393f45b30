"""FP64 restatement of ``CsRss::reconstruct`` (strategy.rs:782-891) including
the reader's placement (reader.rs:225-468) -- test infrastructure only.

Input: headers (a numpy structured array with the fields of
okscuda_acq_header) and the flat complex sample array, as the C-ABI takes
them.  Paths are relative to the reference project's crates/.
"""
from __future__ import annotations

import numpy as np

from oracle import cs_fp64 as o64

NOISE = 1 << 18
REVERSE = 1 << 21
PHASECORR = 1 << 23
NON_IMAGE = (1 << 18) | (1 << 23) | (1 << 22) | (1 << 27) | (1 << 25) | (1 << 26) | (1 << 28)


def _acq(headers, data, i):
    h = headers[i]
    n = int(h["active_channels"]) * int(h["number_of_samples"])
    o = int(h["data_offset"])
    return np.asarray(data[o:o + n], dtype=np.complex128).reshape(int(h["active_channels"]),
                                                                  int(h["number_of_samples"]))


def read_kspace_with_mask(headers, data, encoded, ky_center, kz_center, preprocess):
    """openkspace-io/src/ismrmrd/reader.rs:225-468."""
    img = [i for i in range(len(headers)) if (int(headers[i]["flags"]) & NON_IMAGE) == 0]
    if not img:
        raise ValueError("no image acquisitions found")
    max_ky = max(int(headers[i]["kspace_encode_step_1"]) for i in img)
    max_kz = max(int(headers[i]["kspace_encode_step_2"]) for i in img)
    max_slice = max(int(headers[i]["slice"]) for i in img)
    max_samples = max(int(headers[i]["number_of_samples"]) for i in img)
    nc = max(int(headers[i]["active_channels"]) for i in img)
    if nc == 0:
        raise ValueError("active_channels (0)")
    use_slice = max_kz == 0 and max_slice > 0
    nx = max(encoded[0], max_samples)
    ny = max(encoded[1], max_ky + 1, 1)
    nz = max(max_slice + 1, 1) if use_slice else max(encoded[2], max_kz + 1, 1)
    k = np.zeros((nc, nz, ny, nx), np.complex128)
    filled = np.zeros((nz, ny, nx), bool)
    ky_off = ny // 2 - ky_center
    kz_off = 0 if use_slice else nz // 2 - kz_center
    for i in img:
        h = {n: int(headers[i][n]) for n in headers.dtype.names}
        d = preprocess(_acq(headers, data, i), h)
        ky = h["kspace_encode_step_1"] + ky_off
        kz = (h["slice"] if use_slice else h["kspace_encode_step_2"]) + kz_off
        if ky < 0 or ky >= ny or kz < 0 or kz >= nz:
            continue
        ns = d.shape[1]
        dpre, dpost = h["discard_pre"], h["discard_post"]
        keep = max(ns - (dpre + dpost), 0)
        cs = h["center_sample"]
        dst = max(nx // 2 - (cs - dpre), 0) if (cs > 0 and cs >= dpre) else max(nx - keep, 0) // 2
        src_len = min(keep, max(ns - dpre, 0))
        length = min(src_len, max(nx - dst, 0))
        if length == 0:
            continue
        if filled[kz, ky, dst + length // 2]:
            continue                                    # first wins
        seg = d[:, dpre:dpre + length]
        if h["flags"] & REVERSE:
            seg = seg[:, ::-1]
        ncf = min(d.shape[0], nc)
        k[:ncf, kz, ky, dst:dst + length] = seg[:ncf]
        filled[kz, ky, dst:dst + length] = True
    return k, filled


def csrss_reconstruct(headers, data, encoded, recon, ky_center, kz_center=0, iters=60, lam=0.01,
                      remove_oversampling=True, prewhiten=True, fft_mode="auto", crop=True, phase_correct=True,
                      workers=1):
    noise = [_acq(headers, data, i) for i in range(len(headers)) if int(headers[i]["flags"]) & NOISE]
    w = o64.prewhitener_from_noise(noise) if prewhiten else None
    pc = {}
    if phase_correct:                                   # strategy.rs:790-794
        pc = o64.phase_corrector_from_acqs(
            [(int(headers[i]["slice"]), int(headers[i]["segment"]), _acq(headers, data, i))
             for i in range(len(headers)) if (int(headers[i]["flags"]) & NOISE) == 0
             and int(headers[i]["flags"]) & PHASECORR])
    enc_x, rec_x = encoded[0], recon[0]
    os_ok = remove_oversampling and o64.oversampling_ratio(enc_x, rec_x) is not None

    def preprocess(d, h):
        if w is not None and d.shape[0] == w.shape[0]:
            d = o64.prewhiten_apply(w, d)               # prewhiten.rs:118-142
        if pc:
            d = o64.phase_correct_apply(pc, d, h["slice"], h["segment"])   # phasecorr.rs:141-168
        if os_ok and d.shape[1] == enc_x:
            d = o64.oversampling_apply(d, enc_x, rec_x)  # oversampling.rs:103-155
            h["center_sample"] = rec_x // 2
            h["discard_pre"] = 0
            h["discard_post"] = 0
        return d

    k, filled = read_kspace_with_mask(headers, data, encoded, ky_center, kz_center, preprocess)
    img = [i for i in range(len(headers)) if (int(headers[i]["flags"]) & NON_IMAGE) == 0]
    three_d = fft_mode == "3d" or (fft_mode == "auto" and any(int(headers[i]["kspace_encode_step_2"]) > 0
                                                              for i in img))
    return o64.csrss_from_kspace(k, filled, iters, lam, three_d=three_d,
                                 recon_matrix=tuple(recon) if crop else None, workers=workers)
