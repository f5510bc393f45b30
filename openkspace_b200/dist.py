"""Multi-GPU host logic: one process per GPU, slices sharded across ranks.

The per-coil ``cs`` path has no exchange between (slice, coil) solves
(strategy.rs:850-869), so ranks split the slices of a volume and solve their
share independently; the only communication is the timing reduction (max over
ranks) and gathering the magnitude slices to rank 0.  Works with any
torch.distributed backend (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous balanced share [start, stop) of n items for `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Max of a per-rank scalar (e.g. elapsed ms) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_slices(local: np.ndarray, n_total: int, dist=None, device="cpu") -> np.ndarray | None:
    """Gathers each rank's slices ([n_local, ...] float32, in rank order) into
    [n_total, ...] on rank 0 (None elsewhere)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    shape = local.shape[1:]
    counts = [shard_range(n_total, r, world) for r in range(world)]
    maxn = max(b - a for a, b in counts)
    buf = np.zeros((maxn,) + shape, np.float32)
    buf[:local.shape[0]] = local
    t = torch.from_numpy(buf).to(device)
    parts = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, parts, dst=0)
    if rank != 0:
        return None
    out = np.zeros((n_total,) + shape, np.float32)
    for r, (a, b) in enumerate(counts):
        out[a:b] = parts[r].cpu().numpy()[:b - a]
    return out
