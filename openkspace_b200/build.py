"""Build ``openkspace_b200/libokscuda.so`` (sm_100a) in-tree with nvcc, and
``libokscuda_bounds.so``: the same sources with -DOKS_BOUNDS_CHECK (every
exchange and staging buffer index range-checked into a device error word;
used by the tests only).

``python -m openkspace_b200.build [--verbose] [--force]``.  A library is
rebuilt when any source under ``csrc/`` or ``include/`` is newer than it.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libokscuda.so")
BOUNDS_LIB = os.path.join(HERE, "libokscuda_bounds.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps() -> list[str]:
    return (sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")) + [os.path.abspath(__file__)])


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(p) > t for p in _deps())


def _compile(lib: str, objdir: str, defines: list[str], verbose: bool):
    """(output library, object files, running nvcc processes)."""
    os.makedirs(objdir, exist_ok=True)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *defines, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    return lib, objs, procs


def build(verbose: bool = False, force: bool = False, bounds: bool = True) -> str:
    jobs = []
    if force or needs_build(LIB):
        jobs.append(_compile(LIB, os.path.join(HERE, "_build"), [], verbose))
    if bounds and (force or needs_build(BOUNDS_LIB)):
        jobs.append(_compile(BOUNDS_LIB, os.path.join(HERE, "_build_bounds"), ["-DOKS_BOUNDS_CHECK"], verbose))
    failed = False
    for lib, objs, procs in jobs:
        for src, p in procs:
            out, _ = p.communicate()
            if verbose or p.returncode != 0:
                sys.stdout.write(out.decode(errors="replace"))
            if p.returncode != 0:
                failed = True
                sys.stderr.write(f"nvcc failed on {src} ({os.path.basename(lib)})\n")
    if failed:
        raise RuntimeError("building libokscuda failed")
    for lib, objs, _ in jobs:
        tmp = lib + ".tmp"
        subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
        os.replace(tmp, lib)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
