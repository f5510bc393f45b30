"""FISTA-CS benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plain|volume|precision]

A step is one pass of the hot path over one batch of synthetic input:
  plain      one 8-coil 256 x 256 slice (R = 4 + 24 centre lines, 50 iterations,
             lambda 0.01) through okscuda_cs_slice
  volume     the same slice size, 36 slices per step in one batched launch
value = slices/s with inputs resident in HBM; e2e = the same through the
public API with pinned host buffers copied in and the RSS copied out inside
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
    dominant = "k_fista_col"

    def dominant_bytes_per_launch(self):
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


WORKLOADS = {"plain": lambda: PlainWorkload(1), "volume": lambda: PlainWorkload(36)}


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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
    line = {"impl": "reference", "metric": "FISTA-CS slices/s (CPU restatement of the reference)",
            "value": value, "unit": "slices/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "dtype": "c64", "data": "synthetic", "config": wl.config(),
            "cpu_baseline": {"value": value, "unit": "slices/s", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    wl = WORKLOADS[args.workload]()

    if args.impl == "reference":
        run_reference(args, wl, rank)
        return

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

    units = wl.units * args.steps * world
    value = units / (ms / 1e3)
    e2e_value = units / (ms_e2e / 1e3)
    hbm, peak_kind = peaks()
    dom_ms, dom_n = prof.get(wl.dominant, (0.0, 0))
    per_launch_s = (dom_ms / max(dom_n, 1)) / 1e3
    achieved = wl.dominant_bytes_per_launch() / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    launches = int(sum(n for _, n in prof.values()))

    if rank != 0:
        return
    h2d, d2h = wl.e2e_bytes()
    line = {
        "metric": "FISTA-CS slices/s at NRMSE<=1e-4 vs FP64",
        "value": value, "unit": "slices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic (seeded phantom/coils/noise/masks)",
        "config": {**wl.config(), "parallelism": f"replicas x{world} (slices sharded, no collective)",
                   "l2": "flushed between steps" if flush is not None else "inputs larger than L2"},
        "e2e": {"value": e2e_value, "unit": "slices/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof.items()},
        "roofline": {"bound": "hbm", "kernel": wl.dominant, "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                     "model": "state model: 40 B per pixel per coil per iteration"},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        nthreads = 1
        dt, u, sample = wl.cpu_sample(nthreads)
        line["cpu_baseline"] = {"value": u / dt, "unit": "slices/s", "cores": nthreads, "kind": "port",
                                "sample": sample}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
