"""FISTA-CS benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload precision|plain|volume|batched|served] [--row-engine simt|tc]

A step is one pass of the hot path over one batch of synthetic input:
  precision  (default) 36 slices x 15 coils, 640 (2x oversampled) x 368, R = 4 with an
             8 % centre, correlated noise, 120 iterations, lambda 0.005: the whole
             CsRss pipeline (noise fit, prewhitening, oversampling removal,
             placement, FISTA on the 368 x 640 grid, RSS, crop); the line also
             carries a short run with the other readout engine and a served-vs-plain
             measurement
  plain      one 8-coil 256 x 256 slice (R = 4 + 24 centre lines, 50 iterations)
  volume     36 slices of the plain size in one batched launch
  batched    64 slices of uneven size, coils, R and iterations in one okscuda_cs_batch
  volume3d   32 coils, 256 x 256 x 192 3-D Cartesian, R = 6, 80 iterations: the
             CsRss 3-D path (kz IFFT, 192 x 32 slice solves, RSS)
  served     Poisson arrivals through the request server beside the plain drop-in
  fft        the centred 2-D FFT alone: 1024 coil planes of 368 x 640 in place
             (the row and column transform kernels; metric planes/s);
             --fft-shape NYxNX another plane shape at the same bytes per step
value = slices/s with inputs resident in HBM; e2e = the same through the
public API with pinned host buffers copied in and the result copied out inside
the timed region.  Multi-GPU: one process per GPU, every rank solves its own
slices (no data-path collective; weak scaling).  ``--impl reference`` times
the CPU restatement of the reference (oracle/cs_ref.c; the Rust reference
cannot be built here) on a bounded sample with every host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tc_peak():
    """Dense bf16 tensor peak in TFLOP/s: the sustained figure (the tensor-core
    DFTs run inside a seconds-long step)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured (sustained)"
    return 1400.0, "fallback (sustained)"


# --------------------------------------------------------------- workloads
class PlainWorkload:
    """8 coils, 256 x 256, R = 4 + 24 centre lines, lambda 0.01, 50 iterations."""
    name = "plain"

    def __init__(self, nslices: int = 1):
        from openkspace_b200 import synth
        self.nslices = nslices
        sl = [synth.plain_slice(z) for z in range(nslices)]
        self.nc, self.ny, self.nx = sl[0].kspace.shape
        self.iters, self.lam = 50, 0.01
        self.k = np.ascontiguousarray(np.stack([s.kspace for s in sl], axis=1))   # [nc, nz, ny, nx]
        self.mask = np.stack([s.mask2d for s in sl]).astype(np.uint8)             # [nz, ny, nx]
        self.units = nslices

    def config(self):
        return {"workload": ("plain_slice" if self.nslices == 1 else f"slice_volume_x{self.nslices}")
                + f"_{self.nc}c_{self.ny}x{self.nx}_I{self.iters}",
                "coils": self.nc, "ny": self.ny, "nx": self.nx, "slices_per_step": self.nslices,
                "iters": self.iters, "lambda": self.lam, "mask": "ky-only R=4 + 24 centre lines"}

    def input_bytes(self):
        return self.k.nbytes

    # state-model algorithmic bytes of the fused FISTA kernel per launch:
    # 40 B per pixel per coil per iteration (read z, x, y; write x', z')
    dominant = ("k_fista_col_reg", "k_fista_col")   # register form where a plan exists
    bytes_model = "state model: 40 B per pixel per coil per iteration (read z, x, y; write x', z')"

    def dominant_bytes_per_step(self):
        return 40.0 * self.ny * self.nx * self.nc * self.iters * self.nslices

    def prepare(self, ctx):
        self.ctx = ctx
        self.d_k = ctx.to_device(self.k)
        self.d_out = ctx.empty((self.nslices, self.ny, self.nx), np.float32)
        self.d_coils = ctx.empty(self.k.shape)
        import torch
        self.h_k = torch.from_numpy(self.k.view(np.float32)).pin_memory()
        self.h_out = torch.empty((self.nslices, self.ny, self.nx), dtype=torch.float32).pin_memory()

    def step_device(self):
        c = self.ctx
        c.check(c.lib.okscuda_cs_volume(c.handle, self.d_k.ptr, self.mask.ctypes.data, self.nc, self.nslices,
                                        self.ny, self.nx, self.iters, self.lam, self.ny, self.nx,
                                        self.d_out.ptr, self.d_coils.ptr))

    def step_e2e(self):
        c = self.ctx
        c.check(c.lib.okscuda_upload(c.handle, self.d_k.ptr, self.h_k.data_ptr(), self.k.nbytes))
        self.step_device()
        c.check(c.lib.okscuda_download(c.handle, self.h_out.data_ptr(), self.d_out.ptr, self.h_out.numel() * 4))

    def e2e_bytes(self):
        return self.k.nbytes, self.nslices * self.ny * self.nx * 4

    def cpu_sample(self, nthreads):
        """(seconds, units) for a bounded CPU sample: whole slices, all coils."""
        from oracle import csref
        nz = max(1, min(self.nslices, nthreads // 2 or 1))
        t = time.perf_counter()
        csref.csrss(self.k[:, :nz], self.mask[:nz].astype(bool), self.iters, self.lam, nthreads=nthreads)
        return time.perf_counter() - t, nz, f"{nz} slice(s) x {self.nc} coils x {self.iters} iterations"


class PrecisionWorkload:
    """15 coils, 640 (readout, 2x oversampled) x 368 ky, 36 slices, R = 4 with
    an 8 % centre, 256 noise samples per coil from a covariance of condition
    number 50, lambda 0.005, 120 iterations: the whole CsRss pipeline
    (FP64 noise fit, prewhitening, oversampling removal, placement, FISTA at
    the reference's 368 x 640 grid with partial-row masks, RSS, crop to 320)."""
    name = "precision"
    # the 2-D engine runs as one CUDA graph per call (all chunks and
    # iterations); without graphs its row pass is the largest kernel
    dominant = ("k2d_graph", "k2d_row_reg", "k2d_row")
    bytes_model = ("2-D engine, column + row pass per problem and iteration: column pass reads S and writes S "
                   "on the sampled kx columns (fraction f_c) and reads y on the sampled (ky, kx) points "
                   "(f_c f_r); row pass reads S (f_c), Z~, X~ and writes X~, Z~, S (f_c): "
                   "8 (6 f_c + 4 + f_c f_r) B per pixel; init passes and the demodulated copy added")

    def __init__(self, nz: int = 36, iters: int = 120):
        from openkspace_b200 import synth
        from openkspace_b200.strategy import CsRss, oversampled_acquisitions
        self.vol = synth.oversampled_volume(nz=nz)
        self.acqs = oversampled_acquisitions(self.vol)
        self.iters = iters
        self.strategy = CsRss(iters=iters, lambda_=0.005)
        self.nz, self.nc = nz, self.vol.lines.shape[2]
        self.ny, self.nx = self.vol.ny, self.vol.enc_x
        self.units = nz

    def config(self):
        return {"workload": f"precision_{self.nc}c_{self.vol.enc_x}x{self.ny}_os2_{self.nz}slices_I{self.iters}",
                "coils": self.nc, "slices_per_step": self.nz, "readout": self.vol.enc_x, "ky": self.ny,
                "recon_x": self.vol.rec_x, "fista_grid": f"{self.ny}x{self.nx}", "iters": self.iters, "lambda": 0.005,
                "mask": "ky R=4 + 8% centre; rows partial in kx after oversampling removal",
                "noise": "256 samples/coil, cond(Psi)=50", "pipeline": "CsRss (strategy.rs:782-891)"}

    def input_bytes(self):
        return self.acqs.data.nbytes

    def dominant_bytes_per_step(self, kernel=None):
        npx = self.ny * self.nx * self.nc * self.nz
        if kernel in (None, "k2d_graph"):
            f_c = self.vol.rec_x / self.nx
            f_r = len(self.vol.ky_index[0]) / self.ny
            per_iter = 8.0 * (6 * f_c + 4 + f_c * f_r)
            init = 8.0 * (2 * f_c + f_c * f_r) + 8.0 * (2 * f_c + 2)
            return (per_iter * self.iters + init + 16.0) * npx
        # k2d_row per problem: the init pass reads S, writes X~, Z~, S (32 B
        # per pixel); every iteration reads S, Z~, X~ and writes X~, Z~, S (48 B)
        return (48.0 * self.iters + 32.0) * npx

    tc_flops_model = ("tensor-core row DFTs: per problem and row pass (iterations + init), F_x^H over the "
                      "rec_x sampled kx columns and F_x back onto them, each 3 bf16 products of "
                      "2 * ny * (2 rec_x) * (2 nx) FLOPs")

    def tc_flops_per_step(self):
        per_gemm = 3 * 2.0 * self.ny * (2 * self.vol.rec_x) * (2 * self.nx)
        return 2 * per_gemm * (self.iters + 1) * self.nc * self.nz

    def prepare(self, ctx):
        import torch
        self.ctx = ctx
        self.d_data = ctx.to_device(self.acqs.data)
        self.shape = self.strategy.output_shape(ctx, self.acqs)
        self.d_out = ctx.empty(self.shape, np.float32)
        pinned = torch.from_numpy(self.acqs.data.view(np.float32)).pin_memory()
        self._pinned = pinned
        self.acqs.data = pinned.numpy().view(np.complex64)
        self.h_out = torch.empty(self.shape, dtype=torch.float32).pin_memory().numpy()

    def step_device(self):
        self.strategy.reconstruct(self.ctx, self.acqs, device_data=self.d_data, out=self.d_out)

    def step_e2e(self):
        self.strategy.reconstruct(self.ctx, self.acqs, out=self.h_out)

    def e2e_bytes(self):
        return self.acqs.data.nbytes, int(np.prod(self.shape)) * 4

    def cpu_sample(self, nthreads):
        """The same pipeline through the FP32 C restatement for one slice:
        noise fit, prewhitening, oversampling removal and placement of every
        line, then per-coil FISTA + RSS on `ncoil` coils (scaled to 15)."""
        from oracle import csref
        vol = self.vol
        ncoil = max(1, min(self.nc, nthreads if nthreads > 1 else 2))
        t = time.perf_counter()
        w = csref.prewhiten_fit(vol.noise)
        lines = csref.prewhiten_apply(w, vol.lines[0])                      # [n_lines, nc, 640]
        os = csref.oversampling_apply(lines, vol.enc_x, vol.rec_x)           # [n_lines, nc, 320]
        k = np.zeros((self.nc, 1, self.ny, self.nx), np.complex64)
        m = np.zeros((1, self.ny, self.nx), bool)
        x0 = self.nx // 2 - vol.rec_x // 2
        k[:, 0, vol.ky_index[0], x0:x0 + vol.rec_x] = np.transpose(os, (1, 0, 2))
        m[0, vol.ky_index[0], x0:x0 + vol.rec_x] = True
        csref.csrss(k[:ncoil], m, self.iters, 0.005, nthreads=nthreads)
        dt = time.perf_counter() - t
        units = ncoil / self.nc
        return dt, units, f"1 slice: full feeding pipeline + FISTA on {ncoil} of {self.nc} coils (scaled)"


class BatchedWorkload:
    """64 slices of uneven size {256^2, 320^2, 384^2, 368x640}, 8-32 coils,
    R in {2,3,4,6} + 24 centre lines, 30-150 iterations, in one okscuda_cs_batch
    call per step (one register-engine launch per column length, concurrent)."""
    name = "batched"
    dominant = ("k_fista_col_reg",)
    bytes_model = "state model: 40 B per pixel per coil per iteration (read z, x, y; write x', z')"

    def __init__(self, n: int = 64, reqs=None):
        from openkspace_b200 import synth
        self.reqs = reqs if reqs is not None else synth.uneven_requests(n=n)
        self.units = len(self.reqs)

    @classmethod
    def from_files(cls, d):
        """The 64 slices written by _side_inputs."""
        from openkspace_b200 import synth
        meta = json.load(open(os.path.join(d, "reqs.json")))
        reqs = [synth.SliceRequest(np.load(os.path.join(d, f"req{i}_k.npy")),
                                   np.load(os.path.join(d, f"req{i}_m.npy")), int(it), float(lam))
                for i, (it, lam) in enumerate(meta)]
        return cls(reqs=reqs)

    def check_indices(self):
        """One slice per matrix size, the lightest of each (coils x iterations)."""
        best = {}
        for i, r in enumerate(self.reqs):
            key = r.kspace.shape[1:]
            w = r.kspace.shape[0] * r.iters
            if key not in best or w < best[key][0]:
                best[key] = (w, i)
        return sorted(i for _, i in best.values())

    def config(self):
        return {"workload": f"batched_uneven_{self.units}slices", "sizes": "256^2,320^2,384^2,368x640",
                "coils": "U{8..32}", "accel": "{2,3,4,6} + 24 centre", "iters": "U{30..150}", "lambda": 0.01,
                "coil_iters_px_total": int(sum(r.kspace.shape[0] * r.iters * r.kspace.shape[1] * r.kspace.shape[2]
                                               for r in self.reqs))}

    def input_bytes(self):
        return sum(r.kspace.nbytes for r in self.reqs)

    def dominant_bytes_per_step(self):
        return 40.0 * sum(r.kspace.shape[0] * r.iters * r.kspace.shape[1] * r.kspace.shape[2] for r in self.reqs)

    def prepare(self, ctx):
        import torch
        self.ctx = ctx
        self.d_k = [ctx.to_device(r.kspace) for r in self.reqs]
        self.masks = [np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1) for r in self.reqs]
        self.d_out = [ctx.empty(r.kspace.shape[1:], np.float32) for r in self.reqs]
        self.h_k = [torch.from_numpy(r.kspace.view(np.float32)).pin_memory() for r in self.reqs]
        self.h_out = [torch.empty(r.kspace.shape[1:], dtype=torch.float32).pin_memory() for r in self.reqs]
        self.args = [(d, m, r.iters, r.lam) for d, m, r in zip(self.d_k, self.masks, self.reqs)]

    def step_device(self):
        self.ctx.cs_batch(self.args, outs=self.d_out)

    def step_e2e(self):
        c = self.ctx
        for d, h in zip(self.d_k, self.h_k):
            c.check(c.lib.okscuda_upload(c.handle, d.ptr, h.data_ptr(), d.nbytes))
        self.step_device()
        for d, h in zip(self.d_out, self.h_out):
            c.check(c.lib.okscuda_download(c.handle, h.data_ptr(), d.ptr, d.nbytes))

    def e2e_bytes(self):
        return self.input_bytes(), sum(int(np.prod(r.kspace.shape[1:])) * 4 for r in self.reqs)

    def cpu_sample(self, nthreads):
        from oracle import csref
        r = min(self.reqs, key=lambda r: r.kspace.shape[0] * r.iters * r.kspace.size)
        ncoil = max(1, min(r.kspace.shape[0], nthreads if nthreads > 1 else 2))
        m = np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1)
        t = time.perf_counter()
        csref.csrss(r.kspace[:ncoil, None], m[None], r.iters, r.lam, nthreads=nthreads)
        dt = time.perf_counter() - t
        # scale by work: the whole batch's coil-iteration-pixels over the sample's
        work = sum(q.kspace.shape[0] * q.iters * q.kspace.shape[1] * q.kspace.shape[2] for q in self.reqs)
        sample = ncoil * r.iters * r.kspace.shape[1] * r.kspace.shape[2]
        return dt, self.units * sample / work, f"{ncoil} coils of the lightest slice, scaled by coil-iteration-pixels"


class Volume3dWorkload:
    """32 coils, 256 x 256 x 192 (kz) 3-D Cartesian, ky-only R = 6 with 24
    centre lines (every kz partition), 80 iterations, lambda 0.01: the CsRss
    3-D path -- placement, centred IFFT along kz, then 192 x 32 per-slice
    FISTA solves through the column engine, RSS, crop."""
    name = "volume3d"
    dominant = ("k_fista_col_reg", "k_fista_col")
    bytes_model = "state model: 40 B per pixel per coil per iteration (read z, x, y; write x', z')"

    def __init__(self, nz: int = 192, nc: int = 32, iters: int = 80, data=None):
        from openkspace_b200 import synth
        from openkspace_b200.strategy import CsRss, cartesian3d_acquisitions
        self.k, self.mask_rows = data if data is not None else synth.volume_3d(nc=nc, nz=nz)
        self.acqs = cartesian3d_acquisitions(self.k, self.mask_rows)
        self.strategy = CsRss(iters=iters, lambda_=0.01)
        self.nc, self.nz, self.ny, self.nx = self.k.shape
        self.iters = iters
        self.units = nz

    @classmethod
    def from_files(cls, d):
        """The volume written by _side_inputs."""
        k = np.load(os.path.join(d, "vol_k.npy"))
        m = np.load(os.path.join(d, "vol_m.npy"))
        return cls(nz=k.shape[1], nc=k.shape[0], data=(k, m))

    def config(self):
        return {"workload": f"cartesian3d_{self.nc}c_{self.ny}x{self.nx}x{self.nz}_R6_I{self.iters}",
                "coils": self.nc, "slices_per_step": self.nz, "ny": self.ny, "nx": self.nx, "nz": self.nz,
                "iters": self.iters, "lambda": 0.01, "mask": "ky-only R=6 + 24 centre lines, all kz",
                "pipeline": "CsRss 3-D (strategy.rs:782-891: kz IFFT fft.rs:52-84, per-slice FISTA, RSS)"}

    def input_bytes(self):
        return self.acqs.data.nbytes

    def dominant_bytes_per_step(self):
        return 40.0 * self.ny * self.nx * self.nc * self.nz * self.iters

    def prepare(self, ctx):
        import torch
        self.ctx = ctx
        self.d_data = ctx.to_device(self.acqs.data)
        self.shape = self.strategy.output_shape(ctx, self.acqs)
        self.d_out = ctx.empty(self.shape, np.float32)
        pinned = torch.from_numpy(self.acqs.data.view(np.float32)).pin_memory()
        self._pinned = pinned
        self.acqs.data = pinned.numpy().view(np.complex64)
        self.h_out = torch.empty(self.shape, dtype=torch.float32).pin_memory().numpy()
        self.k_cpu = np.ascontiguousarray(self.k[:2])   # the one-core CPU sample needs two coils
        del self.k   # the acquisition set holds the samples from here on

    def step_device(self):
        self.strategy.reconstruct(self.ctx, self.acqs, device_data=self.d_data, out=self.d_out)

    def step_e2e(self):
        self.strategy.reconstruct(self.ctx, self.acqs, out=self.h_out)

    def e2e_bytes(self):
        return self.acqs.data.nbytes, int(np.prod(self.shape)) * 4

    def cpu_sample(self, nthreads):
        """The FP32 C restatement on one kz-decoupled slice: `ncoil` coils of
        the placed k-space, centred IFFT along kz, FISTA + RSS (scaled to 32)."""
        from oracle import csref
        k = getattr(self, "k", None)
        if k is None:
            k = self.k_cpu
        m = self.mask_rows
        ncoil = max(1, min(k.shape[0], nthreads if nthreads > 1 else 2))
        t = time.perf_counter()
        kz = csref.ifft1_axis(k[:ncoil], 1)[:, :1]                           # [ncoil, 1, ny, nx]
        mask = np.repeat(m[:, None], self.nx, 1)[None]
        csref.csrss(np.ascontiguousarray(kz), mask, self.iters, 0.01, nthreads=nthreads)
        dt = time.perf_counter() - t
        return dt, ncoil / self.nc, f"1 slice: kz IFFT of {ncoil} of {self.nc} coils + FISTA + RSS (scaled)"


class FftWorkload:
    """The centred 2-D FFT of cs.rs:141-178 on a batch of coil planes of the
    precision configuration's encoded size (368 ky x 640 readout), in place:
    one register-resident row pass (length 640) and one column pass (length
    368), each reading and writing every plane once."""
    name = "fft"
    metric = "centred 2-D FFT coil planes/s (relative L2 <= 1e-5 vs FP64)"
    unit = "planes/s"
    data = "synthetic (seeded complex Gaussian planes)"
    dominant = ("k_col_xform", "k_row_xform")
    bytes_model = "16 B per pixel per pass (read + write complex64)"

    def __init__(self, nplanes: int = 1024, ny: int = 368, nx: int = 640):
        self.nplanes, self.ny, self.nx = nplanes, ny, nx
        self.units = nplanes

    def config(self):
        return {"workload": f"centred_fft2_{self.nplanes}x{self.ny}x{self.nx}", "planes_per_step": self.nplanes,
                "ny": self.ny, "nx": self.nx, "direction": "forward, in place",
                "unit": "one coil plane of the precision configuration's encoded size"}

    def input_bytes(self):
        return self.nplanes * self.ny * self.nx * 8

    def dominant_bytes_per_step(self, kernel=None):
        return 16.0 * self.nplanes * self.ny * self.nx

    def prepare(self, ctx):
        import torch
        self.ctx = ctx
        g = torch.Generator(device="cuda").manual_seed(7)
        self.d = torch.randn((self.nplanes, self.ny, self.nx), dtype=torch.complex64, device="cuda", generator=g)
        self.h_in = self.d.cpu().pin_memory()
        self.h_out = torch.empty_like(self.h_in).pin_memory()
        torch.cuda.synchronize()

    def step_device(self):
        c = self.ctx
        c.check(c.lib.okscuda_centred_fft2(c.handle, self.d.data_ptr(), self.nplanes, self.ny, self.nx, 0))

    def step_e2e(self):
        c = self.ctx
        nb = self.input_bytes()
        c.check(c.lib.okscuda_upload(c.handle, self.d.data_ptr(), self.h_in.data_ptr(), nb))
        self.step_device()
        c.check(c.lib.okscuda_download(c.handle, self.h_out.data_ptr(), self.d.data_ptr(), nb))

    def e2e_bytes(self):
        return self.input_bytes(), self.input_bytes()

    def cpu_sample(self, nthreads):
        """The oracle's FP32 centred 2-D FFT (oracle/cs_ref.c) on a few planes."""
        from oracle import csref
        n = 8
        rng = np.random.default_rng(7)
        x = (rng.standard_normal((n, self.ny, self.nx)) + 1j * rng.standard_normal((n, self.ny, self.nx)))
        x = x.astype(np.complex64)
        t = time.perf_counter()
        csref.centred_fft2(x)
        return time.perf_counter() - t, n, f"{n} planes through the oracle's centred FFT2"


def fft_stages(ctx, shapes=((368, 640), (256, 256), (320, 320), (384, 384), (512, 512)), target=1 << 30, reps=5):
    """HBM rate of the row and column passes of the centred 2-D FFT (in place,
    about 1 GiB of planes per shape, above L2): algorithmic 16 B per pixel per
    pass over the device time of each pass's launches."""
    import torch
    hbm, kind = peaks()
    out = {"peak_gbs": hbm, "peak_kind": kind, "bytes_model": "16 B per pixel per pass"}
    for ny, nx in shapes:
        batch = max(1, target // (ny * nx * 8))
        d = torch.zeros((batch, ny, nx), dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        for _ in range(2):
            ctx.check(ctx.lib.okscuda_centred_fft2(ctx.handle, d.data_ptr(), batch, ny, nx, 0))
        ctx.profile(True)
        for _ in range(reps):
            ctx.check(ctx.lib.okscuda_centred_fft2(ctx.handle, d.data_ptr(), batch, ny, nx, 0))
        prof = ctx.profile_read()
        ctx.profile(False)
        rec = {"planes": batch}
        for k, length in (("k_row_xform", nx), ("k_col_xform", ny)):
            ms, n = prof[k]
            gbs = 16.0 * batch * ny * nx / (ms / n / 1e3) / 1e9
            rec[k] = {"length": length, "us_per_launch": 1e3 * ms / n, "achieved_gbs": gbs, "frac": gbs / hbm}
        out[f"{ny}x{nx}"] = rec
        del d
    torch.cuda.synchronize()
    return out


def prewhiten_stage(ctx, nc=15, ns=1280, target=1 << 30, reps=5):
    """HBM rate of the prewhitening apply (prewhiten.rs:118-142) on about 1 GiB
    of raw lines [n][nc][ns] (the precision workload's channel count and
    oversampled readout length): the bulk-copy staged kernel against the
    plain-load one, 16 B per sample per channel (read and write in place)."""
    import torch
    hbm, kind = peaks()
    nacq = max(1, target // (nc * ns * 8))
    d = torch.zeros((nacq, nc, ns), dtype=torch.complex64, device="cuda")
    w = torch.tril(torch.randn((nc, nc), dtype=torch.complex64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(3)))
    torch.cuda.synchronize()
    out = {"peak_gbs": hbm, "peak_kind": kind, "acquisitions": nacq, "channels": nc, "samples": ns,
           "bytes_model": "16 B per sample per channel"}
    for bulk, name in ((1, "k_prewhiten_bulk"), (0, "k_prewhiten_apply")):
        ctx.set_option("prewhiten_bulk", bulk)
        for _ in range(2):
            ctx.check(ctx.lib.okscuda_prewhiten_apply(ctx.handle, w.data_ptr(), d.data_ptr(), nacq, nc, ns))
        ctx.profile(True)
        for _ in range(reps):
            ctx.check(ctx.lib.okscuda_prewhiten_apply(ctx.handle, w.data_ptr(), d.data_ptr(), nacq, nc, ns))
        prof = ctx.profile_read()
        ctx.profile(False)
        ms, n = prof[name]
        gbs = 16.0 * nacq * nc * ns / (ms / n / 1e3) / 1e9
        out[name] = {"us_per_launch": 1e3 * ms / n, "achieved_gbs": gbs, "frac": gbs / hbm}
    ctx.set_option("prewhiten_bulk", -1)
    out["tc_status"] = ctx.tc_status()
    del d
    torch.cuda.synchronize()
    return out


WORKLOADS = {"plain": lambda: PlainWorkload(1), "volume": lambda: PlainWorkload(36),
             "precision": lambda: PrecisionWorkload(36), "batched": lambda: BatchedWorkload(64),
             "volume3d": lambda: Volume3dWorkload(),
             # reduced sizes of the same kernels, for profiler captures only
             "fft": lambda: FftWorkload(),
             "precision_small": lambda: PrecisionWorkload(2, 4), "batched_small": lambda: BatchedWorkload(6),
             "fft_small": lambda: FftWorkload(96)}


def _submit_retry(srv, *a, **kw):
    """srv.submit, retried while admission refuses it (OKS_EAGAIN); returns
    (id, out, refusals)."""
    from openkspace_b200 import OksError, _lib
    refused = 0
    while True:
        try:
            rid, out = srv.submit(*a, **kw)
            return rid, out, refused
        except OksError as e:
            if e.code != _lib.OKS_EAGAIN:
                raise
            refused += 1
            time.sleep(0.0002)


def serving_measure(ctx, rates, seconds, max_requests, mode=0, n_streams=0, volume=None, budget=0):
    """Poisson arrivals of single-slice requests (the serving distribution:
    sizes {256^2, 320^2, 384^2, 368 x 640}, coils U{8..32}, R {2,3,4,6},
    iterations U{30..150}) at several rates through the request server, beside
    the plain per-slice drop-in (okscuda_cs_slice, one at a time, host
    buffers).  Latency = submit -> result on the host.  ``volume`` =
    (DeviceArray [nc, nz, ny, nx] after the kz IFFT, mask [ny, nx], iters,
    lambda): its nz slices are also submitted, in place, as fast as admission
    allows, during the first rate's arrivals (the 3-D workload fed through the
    server beside the serving traffic).  Returns (served per rate, plain,
    volume record or None)."""
    import threading

    import torch
    from openkspace_b200 import synth
    from openkspace_b200.server import Server
    pool = synth.uneven_requests(n=32, workload=3)
    pinned = [torch.from_numpy(r.kspace.view(np.float32)).pin_memory().numpy().view(np.complex64) for r in pool]
    masks = [np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1) for r in pool]
    for k, m, r in zip(pinned, masks, pool):                 # warm-up: every size, iteration count (plans, tables)
        ctx.cs_slice(k, m, r.iters, r.lam)
    # plain per-slice drop-in: three passes over the pool, the median pass rate
    # (one slow host call in a 32-call pass moves a single pass's rate a lot)
    lat, pass_rates = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        for k, m, r in zip(pinned, masks, pool):
            a = time.perf_counter()
            ctx.cs_slice(k, m, r.iters, r.lam)
            lat.append(time.perf_counter() - a)
        pass_rates.append(len(pool) / (time.perf_counter() - t0))
    plain_rate = float(np.median(pass_rates))
    plain = {"slices_per_s": plain_rate, "pass_rates": pass_rates, "p50_ms": 1e3 * float(np.percentile(lat, 50)),
             "p99_ms": 1e3 * float(np.percentile(lat, 99))}
    out, vol_rec = {}, None
    rng = np.random.default_rng(7)
    with Server(ctx, max_inflight=48, n_streams=n_streams, mode=mode, hbm_budget_bytes=budget) as srv:
        for rid0 in range(4):                                   # warm the server path
            i, _ = srv.submit(pinned[rid0], masks[rid0], pool[rid0].iters, pool[rid0].lam)
            srv.wait(i, 120000)
        for ri, rate in enumerate(rates):
            nreq = int(min(max_requests, max(40, rate * seconds)))
            arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
            outs = [np.empty(pool[i % len(pool)].kspace.shape[1:], np.float32) for i in range(nreq)]
            submitted, done, vol_ids = {}, {}, {}
            refusals = [0, 0]
            lock = threading.Lock()
            start = time.perf_counter()

            def submitter():
                for n in range(nreq):
                    j = n % len(pool)
                    while time.perf_counter() - start < arrivals[n]:
                        time.sleep(0.0002)
                    rid, _, nref = _submit_retry(srv, pinned[j], masks[j], pool[j].iters, pool[j].lam, out=outs[n])
                    with lock:
                        submitted[rid] = start + arrivals[n]
                        refusals[0] += nref

            def vol_submitter():
                d, m, iters, lam = volume
                for z in range(d.shape[1]):
                    t = time.perf_counter()
                    rid, _, nref = _submit_retry(srv, None, m, iters, lam, device_slice=(d, z))
                    with lock:
                        vol_ids[rid] = t
                        refusals[1] += nref

            threads = [threading.Thread(target=submitter)]
            with_vol = volume is not None and ri == 0
            if with_vol:
                threads.append(threading.Thread(target=vol_submitter))
            for th in threads:
                th.start()
            nvol = volume[0].shape[1] if with_vol else 0
            while len(done) < nreq + nvol:
                with lock:
                    pend = [r for r in list(submitted) + list(vol_ids) if r not in done]
                for r in pend:
                    if srv.poll(r):
                        done[r] = time.perf_counter()
                time.sleep(0.0002)
            for th in threads:
                th.join()
            span = max(done[r] for r in submitted) - start
            lats = [done[r] - submitted[r] for r in submitted]
            out[str(int(rate))] = {"requests": nreq, "slices_per_s": nreq / span,
                                   "p50_ms": 1e3 * float(np.percentile(lats, 50)),
                                   "p99_ms": 1e3 * float(np.percentile(lats, 99)),
                                   "admission_refusals": refusals[0]}
            if with_vol:
                vspan = max(done[r] for r in vol_ids) - min(vol_ids.values())
                vl = [done[r] - vol_ids[r] for r in vol_ids]
                vol_rec = {"slices": nvol, "slices_per_s": nvol / vspan, "alongside_rate_req_per_s": rate,
                           "p50_ms": 1e3 * float(np.percentile(vl, 50)), "p99_ms": 1e3 * float(np.percentile(vl, 99)),
                           "admission_refusals": refusals[1]}
    return out, plain, vol_rec


def run_serving(args):
    """The serving workload alone: several Poisson rates, both server modes,
    one JSON line."""
    import torch
    from openkspace_b200 import Context
    torch.cuda.set_device(0)
    ctx = Context(0)
    rates = [float(x) for x in args.rates.split(",")]
    out, plain, _ = serving_measure(ctx, rates, args.seconds, args.requests, mode=0)
    out1, _, _ = serving_measure(ctx, [max(rates)], args.seconds, args.requests, mode=1)
    plain_rate = plain["slices_per_s"]
    best = max(out.values(), key=lambda v: v["slices_per_s"])
    line = {"metric": "FISTA-CS slices/s + p50/p99 latency (served vs plain)", "value": best["slices_per_s"],
            "unit": "slices/s", "n_gpus": 1, "higher_is_better": True, "dtype": "c64", "data": "synthetic",
            "config": {"workload": "served_poisson", "rates_req_per_s": rates,
                       "request_distribution": "sizes {256^2,320^2,384^2,368x640}, coils U{8..32}, R {2,3,4,6}, "
                                               "iters U{30..150}, lambda 0.01",
                       "latency": "submit -> result in pinned host memory (host clock)"},
            "served": out, "served_continuous_batching": out1, "plain": plain,
            "served_over_plain": best["slices_per_s"] / plain_rate}
    print(json.dumps(line), flush=True)
    ctx.close()


# ------------------------------------------------------------ measurement
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def run_reference(args, wl, rank):
    """CPU restatement of the reference, every host thread, bounded sample per step."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    times, units = [], 0
    sample = ""
    for i in range(args.warmup + args.steps):
        dt, u, sample = wl.cpu_sample(nthreads)
        if i >= args.warmup:
            times.append(dt)
            units += u
    total = sum(times)
    value = units / total
    vunit = getattr(wl, "unit", "slices/s")
    metric = getattr(wl, "metric", "FISTA-CS slices/s at NRMSE<=1e-4 vs FP64")
    line = {"impl": "reference", "metric": metric, "arm": "CPU restatement of the reference",
            "value": value, "unit": vunit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "dtype": "c64", "data": "synthetic", "config": wl.config(),
            "cpu_baseline": {"value": value, "unit": vunit, "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": vunit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------ kernel roofline records
def precision_kernel_roofline(ctx, wl, hbm, peak_kind):
    """Per-kernel roofline of the 2-D engine's two passes, from one profiled
    step with the CUDA graph off and one stream (every launch timed alone
    with CUDA events on its own stream).  Algorithmic bytes are what each
    pass must move per problem (f_c sampled kx columns, f_r sampled ky rows):
      k2d_row_reg: iteration launches read S (8 f_c), Z~, X~ (16) and write
                   X~, Z~ (16), S (8 f_c): 32 + 16 f_c B per pixel; the
                   initial launch reads S, writes X~, Z~, S: 16 + 16 f_c
      k2d_col_reg: iteration launches read and write S (16 f_c) and read y'
                   on the sampled points (8 f_c f_r); the initial launch
                   reads y' and writes S: 8 f_c + 8 f_c f_r."""
    f_c = wl.vol.rec_x / wl.nx
    f_r = len(wl.vol.ky_index[0]) / wl.ny
    npx = float(wl.ny * wl.nx * wl.nc * wl.nz)
    I = wl.iters
    model = {"k2d_row_reg": ((32 + 16 * f_c) * I + (16 + 16 * f_c)) * npx,
             "k2d_col_reg": ((16 * f_c + 8 * f_c * f_r) * I + (8 * f_c + 8 * f_c * f_r)) * npx}
    ctx.set_option("graph2d", 0)
    ctx.set_option("fista2d_streams", 1)
    try:
        wl.step_device()
        ctx.synchronize()
        ctx.profile(True)
        wl.step_device()
        ctx.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
    finally:
        ctx.set_option("graph2d", 1)
        ctx.set_option("fista2d_streams", 2)
    kernels = {}
    step_ms = sum(v[0] for v in prof.values() if v[1] > 0)   # kernels only (copy scopes count no launch)
    for k, b in model.items():
        ms, n = prof.get(k, (0.0, 0))
        if n == 0 or ms <= 0:
            continue
        gbs = b / (ms / 1e3) / 1e9
        kernels[k] = {"launches": int(n), "us_per_launch": 1e3 * ms / n, "ms_per_step": ms,
                      "share_of_step": ms / step_ms if step_ms > 0 else None,
                      "algorithmic_bytes_per_launch": b / n, "achieved": gbs, "frac": gbs / hbm}
    return kernels, prof


def measure(ctx, wl, stream, steps, warmup, flush_bytes=None):
    """Device and end-to-end rate of one workload (no profiling): a short
    side measurement of the default line."""
    import torch
    flush = None
    if wl.input_bytes() < L2_BYTES:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        wl.step_device()
    wl.step_e2e()
    torch.cuda.synchronize()

    def run(fn, profile=False):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if profile:
            ctx.profile(True)
        torch.cuda.synchronize()
        for a, b in evs:
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.zero_()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        prof = ctx.profile_read() if profile else {}
        if profile:
            ctx.profile(False)
        return sum(a.elapsed_time(b) for a, b in evs), prof

    ms, prof = run(wl.step_device, profile=True)
    ms_e2e, _ = run(wl.step_e2e)
    hbm, kind = peaks()
    dom = next((k for k in wl.dominant if k in prof), wl.dominant[0])
    dms, dn = prof.get(dom, (0.0, 0))
    ach = wl.dominant_bytes_per_step() * steps / (dms / 1e3) / 1e9 if dms > 0 else 0.0
    h2d, d2h = wl.e2e_bytes()
    return {"config": wl.config(), "steps": steps, "ms_per_step": ms / steps,
            "value": wl.units * steps / (ms / 1e3), "unit": "slices/s",
            "e2e": {"value": wl.units * steps / (ms_e2e / 1e3), "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "l2": "flushed between steps" if flush is not None else "inputs larger than L2",
            "gpu_launches": int(sum(n for _, n in prof.values())),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "peak_kind": kind,
                         "unit": "GB/s", "frac": ach / hbm, "model": wl.bytes_model,
                         "note": "register/L2-resident state: the state model can exceed HBM"}}


# ------------------------------------------------------- the CPU baseline leg
def cpu_baseline_leg(wl, gpu_slice0, nthreads, extras):
    """The CPU baseline of the default line and the parity of the timed
    output, both through the oracle (the checker):
      * the FP32 C restatement of the reference (oracle/cs_ref.c) runs slice 0
        of the precision workload -- noise fit, prewhitening, oversampling
        removal, placement, FISTA on all coils, RSS -- on `nthreads` host
        threads: the timed CPU baseline;
      * the GPU's timed output for slice 0 is compared with that output
        (relative L2, the stand-in for the reference `cs` output) and with
        the FP64 oracle of the same pipeline (NRMSE);
      * `extras`: (name, gpu_rss, kspace, mask, iters, lambda) slices of the
        side workloads, checked against the FP64 oracle."""
    from oracle import csref
    from oracle import cs_fp64 as o64
    from oracle import strategy_ref
    from openkspace_b200 import synth
    from openkspace_b200.strategy import oversampled_acquisitions
    vol = wl.vol
    t = time.perf_counter()
    w = csref.prewhiten_fit(vol.noise)
    lines = csref.prewhiten_apply(w, vol.lines[0])
    os_ = csref.oversampling_apply(lines, vol.enc_x, vol.rec_x)
    k = np.zeros((wl.nc, 1, wl.ny, wl.nx), np.complex64)
    m = np.zeros((1, wl.ny, wl.nx), bool)
    x0 = wl.nx // 2 - vol.rec_x // 2
    k[:, 0, vol.ky_index[0], x0:x0 + vol.rec_x] = np.transpose(os_, (1, 0, 2))
    m[0, vol.ky_index[0], x0:x0 + vol.rec_x] = True
    port = csref.csrss(k, m, wl.iters, 0.005, nthreads=nthreads)
    dt = time.perf_counter() - t
    port = o64.maybe_crop(port, (vol.rec_x, wl.ny, 1))
    base = {"value": 1.0 / dt, "unit": "slices/s", "cores": nthreads, "kind": "port",
            "sample": f"slice 0 of the workload: noise fit, prewhitening, oversampling removal and placement of "
                      f"its {vol.lines.shape[1]} lines, FISTA on all {wl.nc} coils ({wl.iters} iterations), RSS, "
                      f"crop; oracle/cs_ref.c on {nthreads} host threads"}
    a1 = oversampled_acquisitions(synth.oversampled_volume(nz=1))    # slice 0: same seeds
    t = time.perf_counter()
    want = strategy_ref.csrss_reconstruct(a1.headers, a1.data, a1.encoded, a1.recon, a1.ky_center, a1.kz_center,
                                          iters=wl.iters, lam=0.005, workers=nthreads)
    t64 = time.perf_counter() - t
    parity = {"slice": 0, "nrmse_vs_fp64": o64.nrmse(gpu_slice0, want[0]),
              "rel_l2_vs_port": o64.nrmse(gpu_slice0, port[0]),
              "port_nrmse_vs_fp64": o64.nrmse(port[0], want[0]), "fp64_oracle_s": t64,
              "tolerance": 1e-4, "image": "RSS magnitude after crop (368 x 320)"}
    checks = {}
    for name, rss, ks, mask, iters, lam in extras:
        x = o64.csrss_from_kspace(ks[:, None], mask[None], iters, lam, workers=nthreads)
        checks[name] = o64.nrmse(rss, x[0])
    parity["side_workloads_nrmse_vs_fp64"] = checks
    return base, parity


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="precision", choices=sorted(WORKLOADS) + ["served"])
    ap.add_argument("--row-engine", default="simt", choices=["simt", "tc"],
                    help="2-D-mask engine readout transforms: FP32 SIMT FFT or tcgen05 3xBF16 DFT")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fft-shape", default="368x640",
                    help="fft workloads: plane shape NYxNX (the column pass runs length NY, the row pass NX)")
    ap.add_argument("--no-extras", action="store_true",
                    help="precision: skip the side measurements (other readout engine, FFT stages, serving, "
                         "configurations 0, 2 and 4)")
    ap.add_argument("--rates", default="50,200,800", help="served: Poisson arrival rates (req/s)")
    ap.add_argument("--seconds", type=float, default=60.0, help="served: arrivals per rate x this many seconds")
    ap.add_argument("--requests", type=int, default=2000, help="served: at most this many requests per rate")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "served":
        if rank == 0 and args.impl == "ours":
            run_serving(args)
        return
    wl = WORKLOADS[args.workload]()
    if wl.name == "fft":
        ny, nx = (int(v) for v in args.fft_shape.lower().split("x"))
        wl = FftWorkload(max(1, wl.nplanes * 368 * 640 // (ny * nx)), ny, nx)   # same bytes per step

    if args.impl == "reference":
        run_reference(args, wl, rank)
        return

    extras = wl.name == "precision" and not args.no_extras and world == 1 and rank == 0
    side_inputs = None
    if extras:
        # the side workloads' synthetic inputs are generated in a separate
        # process (spawned before the first GPU call) while this one measures
        import multiprocessing as mp
        # two math-library threads in the generator (the spawned process reads
        # these at its numpy import), so that it does not compete with the
        # host side of the timed end-to-end calls for every core
        saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
        for k in saved:
            os.environ[k] = "2"
        side_pool = mp.get_context("spawn").Pool(1)
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        side_dir = tempfile.mkdtemp()
        side_inputs = side_pool.apply_async(_side_inputs, (side_dir,))

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from openkspace_b200 import Context
    ctx = Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_option("row_engine", 1 if args.row_engine == "tc" else 0)
    wl.prepare(ctx)
    flush = None
    if wl.input_bytes() < L2_BYTES:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(step_fn, k, profile=False):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        if profile:
            ctx.profile(True)
        barrier()
        for a, b in evs:
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.zero_()
            a.record(stream)
            step_fn()
            b.record(stream)
        barrier()
        prof = ctx.profile_read() if profile else None
        if profile:
            ctx.profile(False)
        ms = sum(a.elapsed_time(b) for a, b in evs)
        if dist is not None:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, prof

    for _ in range(args.warmup):
        wl.step_device()
    for _ in range(2):
        wl.step_e2e()
    barrier()

    clocks = ClockSampler(local)
    clocks.start()
    ms, prof = timed(wl.step_device, args.steps, profile=True)
    ms_e2e, _ = timed(wl.step_e2e, args.steps)
    clk = clocks.stop()
    gpu_slice0 = None
    if wl.name == "precision":
        gpu_slice0 = wl.d_out.to_host()[0]       # slice 0 of the last timed step's output

    units = wl.units * args.steps * world
    value = units / (ms / 1e3)
    e2e_value = units / (ms_e2e / 1e3)
    hbm, peak_kind = peaks()
    launches = int(sum(n for _, n in prof.values()))
    h2d, d2h = wl.e2e_bytes()
    metric = getattr(wl, "metric", "FISTA-CS slices/s at NRMSE<=1e-4 vs FP64")
    vunit = getattr(wl, "unit", "slices/s")
    tfile = os.path.join(ROOT, "profiles", "dram_traffic.json")   # per-launch ncu DRAM bytes, by workload
    traffic_tab = json.load(open(tfile)) if os.path.exists(tfile) else {}

    if wl.name == "precision" and args.row_engine == "simt":
        # the dominant kernel's own roofline (non-graph profiled step); the
        # whole engine against the state model beside it
        kernels, prof_ng = precision_kernel_roofline(ctx, wl, hbm, peak_kind)
        dom_name = max(kernels, key=lambda k: kernels[k]["ms_per_step"]) if kernels else "k2d_row_reg"
        kd = kernels.get(dom_name, {"achieved": 0.0, "frac": 0.0})
        t = traffic_tab.get("precision_chunk_12x368x640", {}).get(dom_name)
        graph_ms = prof.get("k2d_graph", (ms, 1))[0]
        state_b = 40.0 * wl.ny * wl.nx * wl.nc * wl.nz * wl.iters * args.steps
        roofline = {"bound": "hbm", "kernel": dom_name, "achieved": kd["achieved"], "peak": hbm,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": kd["frac"],
                    "traffic": float(t["dram_bytes_per_launch"]) if t else None,
                    "traffic_note": (t or {}).get("note"),
                    "model": precision_kernel_roofline.__doc__.split("Algorithmic bytes", 1)[1].strip(),
                    "timing": "one profiled step with the CUDA graph off and one stream: each launch timed alone",
                    "kernels": kernels,
                    "engine_state_model": {
                        "model": "40 B per pixel per coil per iteration (read z, x, y; write x', z') over the "
                                 "2-D engine's graph time in the timed steps",
                        "achieved": state_b / (graph_ms / 1e3) / 1e9,
                        "frac": state_b / (graph_ms / 1e3) / 1e9 / hbm}}
    else:
        bound, unit, peak, model = "hbm", "GB/s", hbm, wl.bytes_model
        dom_name = next((k for k in wl.dominant if k in prof), wl.dominant[0])
        dom_ms, dom_n = prof.get(dom_name, (0.0, 0))
        dbytes = (wl.dominant_bytes_per_step(dom_name) if wl.name in ("precision", "fft")
                  else wl.dominant_bytes_per_step())
        achieved = dbytes * args.steps / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
        if wl.name == "precision" and args.row_engine == "tc":
            # tensor-core row DFTs: the tcgen05 FLOPs they issue / their device time
            dom_name = "k_dft_tc"
            dom_ms, dom_n = prof.get(dom_name, (0.0, 0))
            bound, unit = "tensor", "TFLOP/s"
            peak, peak_kind = tc_peak()
            achieved = wl.tc_flops_per_step() * args.steps / (dom_ms / 1e3) / 1e12 if dom_ms > 0 else 0.0
            model = wl.tc_flops_model
        t = traffic_tab.get(wl.config()["workload"], {}).get(dom_name)
        roofline = {"bound": bound, "kernel": dom_name, "achieved": achieved, "peak": peak,
                    "peak_kind": peak_kind, "unit": unit, "frac": achieved / peak,
                    "traffic": float(t) if isinstance(t, (int, float)) else None, "model": model}

    # precision workload: the other readout engine, a few steps, for the
    # SIMT FFT vs tensor-core DFT comparison on the same configuration
    other = None
    if wl.name == "precision" and not args.no_extras:
        other_engine = "simt" if args.row_engine == "tc" else "tc"
        ctx.set_option("row_engine", 1 if other_engine == "tc" else 0)
        wl.step_device()
        k_other = 3
        ms_o, prof_o = timed(wl.step_device, k_other, profile=True)
        ctx.set_option("row_engine", 1 if args.row_engine == "tc" else 0)
        other = {"row_engine": other_engine, "steps": k_other, "ms_per_step": ms_o / k_other,
                 "value": wl.units * k_other * world / (ms_o / 1e3), "unit": "slices/s",
                 "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof_o.items()}}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": metric,
        "value": value, "unit": vunit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": getattr(wl, "data", "synthetic (seeded phantom/coils/noise/masks)"),
        "config": {**wl.config(), "parallelism": f"replicas x{world} (slices sharded, no collective)",
                   "l2": "flushed between steps" if flush is not None else "inputs larger than L2"},
        "e2e": {"value": e2e_value, "unit": vunit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof.items()},
        "roofline": roofline,
        "clocks": clk,
    }
    if wl.name == "precision":
        line["config"]["row_engine"] = ("FP32 SIMT FFT" if args.row_engine == "simt"
                                        else "tcgen05 split-3xBF16 DFT-as-GEMM, FP32 accumulation")
    if other is not None:
        line["other_row_engine"] = other
    side_checks = []
    if extras:
        # the FFT stages on their own: row and column passes of the centred
        # 2-D FFT at the configuration's lengths, against the HBM roofline
        line["fft_stages"] = fft_stages(ctx)
        line["prewhiten_stage"] = prewhiten_stage(ctx)
        # configurations 0, 2 and 4, each a short device + end-to-end measurement
        configs = {}
        pw = PlainWorkload(1)
        pw.prepare(ctx)
        configs["plain_8x256x256_I50"] = measure(ctx, pw, stream, 10, 3)
        rss0 = pw.d_out.to_host()[0]
        side_checks.append(("plain_8x256x256_I50", rss0, pw.k[:, 0], pw.mask[0].astype(bool), pw.iters, pw.lam))
        del pw
        d = side_inputs.get(timeout=1800)
        bw = BatchedWorkload.from_files(d)
        bw.prepare(ctx)
        configs["batched_uneven_64"] = measure(ctx, bw, stream, 5, 3)
        for i in bw.check_indices():
            r = bw.reqs[i]
            side_checks.append((f"batched_uneven_64[{i}] {r.kspace.shape[0]}x{r.kspace.shape[1]}x"
                                f"{r.kspace.shape[2]} I{r.iters}", bw.d_out[i].to_host(), r.kspace,
                                np.repeat(r.mask_rows[:, None], r.kspace.shape[2], 1), r.iters, r.lam))
        del bw
        vw = Volume3dWorkload.from_files(d)
        vw.prepare(ctx)
        configs["cartesian3d_32x256x256x192_I80"] = measure(ctx, vw, stream, 3, 3)
        del vw
        # the metric's served-vs-plain half: Poisson arrivals of the uneven
        # request mix through the request server at three rates, beside the
        # plain per-slice drop-in (host clock, submit -> result on the host);
        # run once the input generator above has finished, so that no other
        # process competes for the host cores the latencies depend on
        sctx = Context(local)
        served, plain, _ = serving_measure(sctx, [50.0, 200.0, 800.0], 20.0, 2000)
        served1, _, _ = serving_measure(sctx, [800.0], 20.0, 2000, mode=1)
        sctx.close()
        cap = max(v["slices_per_s"] for v in served.values())
        line["serving"] = {"served": served, "served_continuous_batching": served1, "plain": plain,
                           "served_over_plain": cap / plain["slices_per_s"],
                           "served_over_plain_note": "served capacity (the saturating rate, 800 req/s) over the "
                                                     "plain drop-in's rate; at 50 and 200 req/s the server keeps up "
                                                     "with the arrivals (compare the latencies)",
                           "requests": "sizes {256^2,320^2,384^2,368x640}, coils U{8..32}, R {2,3,4,6}, "
                                       "iters U{30..150}; up to 2000 requests or 20 s of arrivals per rate; "
                                       "server mode 0 (one stream per request, the default) at every rate, "
                                       "mode 1 (continuous batching) at 800 req/s"}
        # configuration 4 as specified: the kz-decoupled volume's 192 slices
        # fed through the request server beside Poisson serving traffic at
        # 200 req/s, under a 3 GiB HBM admission budget
        vctx = Context(local)
        vk = np.load(os.path.join(d, "vol_k.npy"))
        vm = np.load(os.path.join(d, "vol_m.npy"))
        d_vol = vctx.to_device(vk)
        nc_, nz_, ny_, nx_ = vk.shape
        del vk
        vctx.check(vctx.lib.okscuda_ifft1_kz(vctx.handle, d_vol.ptr, nc_, nz_, ny_, nx_))
        vctx.synchronize()
        mask2d = np.repeat(vm[:, None], nx_, 1)
        served_v, plain_v, vol_rec = serving_measure(vctx, [200.0], 10.0, 2000, volume=(d_vol, mask2d, 80, 0.01),
                                                     budget=3 << 30)
        configs["cartesian3d_served_with_serving_traffic"] = {
            "volume": vol_rec, "serving_traffic": served_v, "plain": plain_v,
            "hbm_budget_bytes": 3 << 30,
            "note": "32 coils x 256 x 256 x 192, kz IFFT on the device, then the 192 slices (80 iterations, "
                    "lambda 0.01) submitted in place (coil stride nz*ny*nx) while Poisson requests of the serving "
                    "distribution arrive at 200 req/s; slices/s from the first volume submit to the last volume "
                    "slice done"}
        del d_vol
        vctx.close()
        side_pool.close()
        import shutil
        shutil.rmtree(side_dir, ignore_errors=True)
        line["configurations"] = configs
    if not args.no_cpu_baseline and wl.name == "precision" and world == 1:
        nthreads = os.cpu_count() or 1
        line["cpu_baseline"], line["parity"] = cpu_baseline_leg(wl, gpu_slice0, nthreads, side_checks)
    elif not args.no_cpu_baseline:
        nthreads = 1
        dt, u, sample = wl.cpu_sample(nthreads)
        line["cpu_baseline"] = {"value": u / dt, "unit": vunit, "cores": nthreads, "kind": "port",
                                "sample": sample}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _side_inputs(tmpdir):
    """Synthetic inputs of configurations 2 (64 uneven slices) and 4 (the
    3-D Cartesian volume), saved as .npy files in tmpdir (run in a spawned
    process while the main one measures)."""
    from openkspace_b200 import synth
    reqs = synth.uneven_requests(n=64)
    for i, r in enumerate(reqs):
        np.save(os.path.join(tmpdir, f"req{i}_k.npy"), r.kspace)
        np.save(os.path.join(tmpdir, f"req{i}_m.npy"), r.mask_rows)
    json.dump([[r.iters, r.lam] for r in reqs], open(os.path.join(tmpdir, "reqs.json"), "w"))
    k, m = synth.volume_3d(nc=32, nz=192)
    np.save(os.path.join(tmpdir, "vol_k.npy"), k)
    np.save(os.path.join(tmpdir, "vol_m.npy"), m)
    return tmpdir


if __name__ == "__main__":
    main()
