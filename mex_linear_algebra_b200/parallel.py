"""Multi-GPU plumbing: one process per GPU over torch.distributed.

The GF(2) work shards without any data exchange: independent products run
as replicas, and a batch of matrices is split across ranks by estimated cost
(each matrix's rank and null space is computed entirely on one GPU).  The
only collectives are timing/bookkeeping: a barrier around timed regions and
the maximum of per-rank times.
"""
from __future__ import annotations

import os

import numpy as np


def world():
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _device_for_backend():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws: int, value: float) -> float:
    if ws == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(ws: int, value: float) -> float:
    if ws == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def batch_cost(shapes) -> np.ndarray:
    """Work estimate of each matrix's elimination: m * n * ceil(n/64)."""
    s = np.asarray(shapes, dtype=np.float64).reshape(-1, 2)
    return s[:, 0] * s[:, 1] * np.ceil(s[:, 1] / 64.0)


def shard_batch(shapes, world_size: int, rank: int) -> np.ndarray:
    """Indices of the matrices rank `rank` owns: greedy longest-processing-
    time assignment by batch_cost, deterministic on every rank."""
    cost = batch_cost(shapes)
    order = np.argsort(-cost, kind="stable")
    load = np.zeros(world_size)
    owner = np.empty(len(cost), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += cost[i]
    return np.nonzero(owner == rank)[0]


def gather_objects(ws: int, obj):
    """Every rank's `obj`, in rank order, on every rank (host objects)."""
    if ws == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * ws
    dist.all_gather_object(out, obj)
    return out


def run_sharded(shapes, ws: int, rank: int, compute):
    """One batch split over the ranks with no data exchange: rank r runs
    ``compute(indices)`` on the matrices ``shard_batch`` gives it (the
    indices into `shapes`) and returns a dict {index: result}; the results
    are gathered on the host of every rank.  Returns (merged results, the
    indices each rank ran).  Raises if a matrix was computed by no rank or
    by two."""
    mine = shard_batch(shapes, ws, rank)
    local = compute(mine)
    parts = gather_objects(ws, (mine.tolist(), local))
    merged, owners = {}, []
    for idx, res in parts:
        owners.append(idx)
        for i in idx:
            if i in merged:
                raise RuntimeError(f"matrix {i} computed by two ranks")
            if i not in res:
                raise RuntimeError(f"matrix {i} has no result from its rank")
            merged[i] = res[i]
    missing = set(range(len(np.asarray(shapes).reshape(-1, 2)))) - set(merged)
    if missing:
        raise RuntimeError(f"{len(missing)} matrices computed by no rank")
    return merged, owners

