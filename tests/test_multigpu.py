"""Multi-process plumbing of the multi-GPU path on CPU (gloo, world size 2):
slab sharding by slice, max-over-ranks timing, gathering of volume slabs.
The GPU path uses the same functions with NCCL (bench.py --gpus N)."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from tomocupy_b200.multigpu import slab_bounds


@pytest.mark.parametrize("nz,ncz,world", [(2048, 32, 8), (10, 2, 2), (7, 2, 4), (3, 8, 2),
                                          (100, 8, 3)])
def test_slab_bounds_cover_rows_once_aligned_and_balanced(nz, ncz, world):
    spans = [slab_bounds(nz, ncz, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == nz
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0
    chunks = [-(-(z1 - z0) // ncz) for z0, z1 in spans]
    assert max(chunks) - min(chunks) <= 1
    assert all(z0 % ncz == 0 for z0, z1 in spans if z1 > z0)  # empty slabs sit at nz


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nz, ncz, n, q):
    import torch.distributed as dist
    from tomocupy_b200.multigpu import barrier, gather_volume, max_over_ranks, slab_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z0, z1 = slab_bounds(nz, ncz, rank, world)
        # stand-in for this rank's reconstruction of rows [z0, z1)
        slab = (torch.arange(z0, z1, dtype=torch.float32)[:, None, None] +
                torch.zeros((1, n, n)))
        t = max_over_ranks(10.0 * (rank + 1))
        barrier()
        vol = gather_volume(slab, nz, ncz)
        if rank == 0:
            want = torch.arange(nz, dtype=torch.float32)[:, None, None] + torch.zeros((1, n, n))
            q.put(("vol", bool(torch.equal(vol, want))))
        else:
            q.put(("none", vol is None))
        q.put(("t", t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nz,ncz", [(10, 2), (3, 4)])
def test_two_ranks_gloo_shard_time_gather(nz, ncz):
    world, n = 2, 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nz, ncz, n, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = [q.get(timeout=10) for _ in range(2 * world)]
    assert ("vol", True) in got and ("none", True) in got
    assert [v for k, v in got if k == "t"] == [20.0, 20.0]
