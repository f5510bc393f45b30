"""Multi-process host logic on CPU (gloo, world size 2): sharding covers every
slice exactly once, the timing reduction takes the max over ranks, and the
gathered volume equals the single-process result (computed by the FP32
restatement, so no GPU is needed)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from openkspace_b200.dist import shard_range


def test_shard_range_covers_everything():
    for n in (0, 1, 5, 36, 37):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = shard_range(n, r, world)
                assert 0 <= a <= b <= n
                seen += list(range(a, b))
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, ret):
    import datetime

    import torch.distributed as dist

    from oracle import csref
    from openkspace_b200.dist import gather_slices, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(3)
    nc, nz, ny, nx = 2, 5, 16, 12
    k = (rng.standard_normal((nc, nz, ny, nx)) + 1j * rng.standard_normal((nc, nz, ny, nx))).astype(np.complex64)
    m = np.zeros((nz, ny, nx), bool)
    m[:, ::2] = True
    a, b = shard_range(nz, rank, world)
    local = csref.csrss(k[:, a:b], m[a:b], 10, 0.02, nthreads=1) if b > a else np.zeros((0, ny, nx), np.float32)
    full = gather_slices(local, nz, dist)
    t = max_over_ranks(10.0 * (rank + 1), dist)
    if rank == 0:
        want = csref.csrss(k, m, 10, 0.02, nthreads=1)
        ret.put((bool(np.array_equal(full, want)), t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_volume():
    ctx = mp.get_context("spawn")
    ret = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ret)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    same, t = ret.get(timeout=5)
    assert same
    assert t == 20.0
