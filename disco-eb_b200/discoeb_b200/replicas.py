"""Several GPUs: one process per GPU, each solving its own replica of the work.

The k-modes and cosmologies of this path are independent, so nothing is exchanged on the data
path: every rank runs its own launches and the ranks only meet to start together and to take
the slowest rank's time (``max_over_ranks``).  ``shard`` splits one set of modes over the
ranks instead (longest-first order kept, modes dealt round-robin so that every rank gets a
similar mix of step counts) for callers who want one cosmology spread over several GPUs.
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def init(backend="nccl", device=None, timeout_s=120):
    """(rank, world, dist or None) from the torchrun environment (RANK, WORLD_SIZE, MASTER_*).
    With one process nothing is initialised and dist is None."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world <= 1:
        return rank, world, None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl" and device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return rank, world, dist


def max_over_ranks(x, dist, device=None):
    """The largest value of x over all ranks (x itself with one process)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def shard(kmodes, rank, world):
    """Indices of the modes of rank ``rank`` out of ``world``: sorted longest-first (largest k),
    then dealt round-robin."""
    order = np.argsort(-np.asarray(kmodes), kind="stable")
    return np.sort(order[rank::world])


def finish(dist):
    """Barrier and tear-down (every rank calls it, in the same order as every collective)."""
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
