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
