"""One process per GPU: rank discovery, z-slab ownership and device-time reduction.

The reconstruction shards without communication on the data path: either every rank
reconstructs its own volume (replicas, weak scaling) or every rank owns a z-slab of one
volume and backprojects it from the full projection set (the slab's voxels need only the
detector rows they project to; each slab is an independent sub-volume problem through
volStart/volEnd).  The only collectives are the barrier around the timed region and the
max-reduction of the per-rank device times.
"""
from __future__ import annotations

import datetime
import os


def env_ranks():
    """(rank, world_size, local_rank) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, device=None, timeout_s: float = 120.0) -> bool:
    """Initialise the default process group when WORLD_SIZE > 1; returns whether it did.
    A short timeout makes ranks that wait for a missing peer end with an error."""
    import torch.distributed as dist

    _, world, _ = env_ranks()
    if world <= 1 or dist.is_initialized():
        return False
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return True


def max_over_ranks(x: float, device) -> float:
    """The maximum of a per-rank value (device times are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def z_slab(nz: int, world: int, rank: int, align: int = 32):
    """[z0, z1) owned by `rank` when `world` ranks split nz planes: slabs are multiples of
    `align` planes (the backprojector's z tile) except the last; ranks beyond the planes
    get an empty range."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    per = -(-nz // world)
    per = -(-per // align) * align
    z0 = min(nz, rank * per)
    return z0, min(nz, z0 + per)
