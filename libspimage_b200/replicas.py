"""Multi-GPU plumbing for independent reconstructions (replicas).

Phase retrieval has no exchange step: random starts and jobs are independent,
so N GPUs run N replicas, one process per GPU.  This module holds the little
host logic that involves more than one rank -- job sharding, the max-over-ranks
timing reduction, gathering results -- over ``torch.distributed`` (NCCL on
GPUs, gloo in the CPU tests).  Nothing here runs on the data path.
"""
from __future__ import annotations

import datetime
import os


def dist_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 300.0) -> bool:
    """Initialises the process group when WORLD_SIZE > 1; returns whether it did."""
    import torch.distributed as dist

    world, _, _ = dist_env()
    if world <= 1 or dist.is_initialized():
        return dist.is_initialized()
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return True


def shard(footprints, world: int, rank: int):
    """Indices of the jobs this rank runs: largest first onto the least-loaded
    rank (ties to the lower rank), identical on every rank."""
    load = [0] * world
    owner = [0] * len(footprints)
    for i in sorted(range(len(footprints)), key=lambda i: (-footprints[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += footprints[i]
    return [i for i in range(len(footprints)) if owner[i] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Largest value over all ranks (the slowest rank's time)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather(obj):
    """Every rank's object, in rank order (host pickles; results only)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
