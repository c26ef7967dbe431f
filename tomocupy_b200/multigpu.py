"""Multi-GPU plumbing: one process per GPU, slices sharded with no exchange.

Every slice (slice pair for fourierrec) is an independent reconstruction, so
N GPUs split the rows of a volume into contiguous slabs aligned to the chunk
size and reconstruct them with no collective on the data path
(GPURec.recon_all on each rank's slab).  Collectives are used only to time
(the maximum of the ranks' device times) and, when a caller wants the whole
volume on one rank, to gather the slabs.  torch.distributed provides the
process group: NCCL on GPUs, gloo on CPU (tests).

The reference runs one process per node with threads and no multi-GPU
reconstruction path; this module is the B200 replacement for running
independent jobs per GPU.
"""
from __future__ import annotations

import torch


def slab_bounds(nz: int, ncz: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [z0, z1) of ``rank``: contiguous, chunk-aligned, balanced to one chunk."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    nchunks = -(-nz // ncz)
    base, extra = divmod(nchunks, world)
    c0 = rank * base + min(rank, extra)
    c1 = c0 + base + (1 if rank < extra else 0)
    return min(nz, c0 * ncz), min(nz, c1 * ncz)


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank number (e.g. a device time in ms) over all ranks."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None) -> None:
    """Device synchronize (if on a GPU) + process barrier."""
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)
    dist = _dist()
    if dist is not None and dist.get_world_size() > 1:
        dist.barrier()
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)


def gather_volume(slab: torch.Tensor, nz: int, ncz: int, dst: int = 0):
    """Assemble the ranks' slabs [z1 - z0, n, n] into the volume [nz, n, n] on ``dst``.

    Slabs go to ``dst`` one rank at a time (point-to-point), so the
    destination never holds more than the volume plus one slab.  Returns the
    volume on ``dst`` and None elsewhere.
    """
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return slab
    rank, world = dist.get_rank(), dist.get_world_size()
    if rank != dst:
        z0, z1 = slab_bounds(nz, ncz, rank, world)
        if z1 > z0:  # empty slabs are neither sent nor received
            dist.send(slab.contiguous(), dst)
        return None
    vol = torch.empty((nz,) + tuple(slab.shape[1:]), dtype=slab.dtype, device=slab.device)
    for r in range(world):
        z0, z1 = slab_bounds(nz, ncz, r, world)
        if r == dst:
            vol[z0:z1] = slab
        elif z1 > z0:
            buf = torch.empty((z1 - z0,) + tuple(slab.shape[1:]), dtype=slab.dtype,
                              device=slab.device)
            dist.recv(buf, r)
            vol[z0:z1] = buf
    return vol
