"""Several GPUs: one process per GPU, each solving its own replica of the work.

The k-modes and cosmologies of this path are independent, so nothing is exchanged on the data
path: every rank runs its own launches and the ranks only meet to start together and to take
the slowest rank's time (``max_over_ranks``).  ``shard`` splits one set of modes over the
ranks instead (longest-first order kept, modes dealt round-robin so that every rank gets a
similar mix of step counts) for callers who want one cosmology spread over several GPUs; the
results come back together with ``gather_rows`` (every rank receives all rows, in the caller's
mode order) or, for integrals over the modes such as C_l, with ``sum_over_ranks`` of each
rank's partial sum.
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


def gather_rows(local, idx, n_total, dist, device=None):
    """The full [n_total, ...] array on every rank from each rank's rows ``local`` [len(idx), ...]
    at positions ``idx`` (a ``shard``).  One process: the rows placed at idx.  The exchange is an
    all_gather of the (padded) rows and their indices; ``device`` is where the collective's
    tensors live (a CUDA device with NCCL, None for the CPU with gloo)."""
    local = np.asarray(local, dtype=np.float64)
    idx = np.asarray(idx, dtype=np.int64)
    if local.shape[0] != idx.shape[0]:
        raise ValueError("local must have one row per index")
    out = np.full((n_total,) + local.shape[1:], np.nan)
    if dist is None:
        out[idx] = local
        return out
    import torch
    world = dist.get_world_size()
    cnt = torch.tensor([idx.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(cnt) for _ in range(world)]
    dist.all_gather(counts, cnt)
    counts = [int(c.item()) for c in counts]
    m = max(counts)
    pad_v = torch.zeros((m,) + local.shape[1:], dtype=torch.float64, device=device)
    pad_v[:idx.shape[0]] = torch.from_numpy(local).to(pad_v.device)
    pad_i = torch.full((m,), -1, dtype=torch.int64, device=device)
    pad_i[:idx.shape[0]] = torch.from_numpy(idx).to(pad_i.device)
    gv = [torch.empty_like(pad_v) for _ in range(world)]
    gi = [torch.empty_like(pad_i) for _ in range(world)]
    dist.all_gather(gv, pad_v)
    dist.all_gather(gi, pad_i)
    seen = np.zeros(n_total, dtype=np.int64)
    for r in range(world):
        ii = gi[r][:counts[r]].cpu().numpy()
        out[ii] = gv[r][:counts[r]].cpu().numpy()
        np.add.at(seen, ii, 1)
    if not np.all(seen == 1):
        raise RuntimeError("the ranks' row indices do not cover every row exactly once")
    return out


def sum_over_ranks(x, dist, device=None):
    """The sum over all ranks of the array x (x itself with one process): the reduction of
    per-rank partial integrals."""
    x = np.asarray(x, dtype=np.float64)
    if dist is None:
        return x.copy()
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x)).to(device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def finish(dist):
    """Barrier and tear-down (every rank calls it, in the same order as every collective)."""
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
