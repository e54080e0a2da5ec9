"""Multi-GPU plumbing: one process per GPU, launched by torch.distributed.run.

The removal path has no data-path collective: a single list does not split without an exchange
step, so N GPUs run N independent replicas (one list each); batched lists and service shards are
partitioned by list / shard. What crosses ranks is only control: a start barrier and the
max-over-ranks of a measured time (the job is as slow as its slowest rank).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def env_ranks() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 120) -> tuple[int, int, int]:
    """Join the process group when the launcher started more than one rank. With NCCL each rank
    binds its own GPU (local rank). A short timeout turns a missing rank into an error."""
    import torch
    import torch.distributed as dist

    world, rank, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        kwargs = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kwargs["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kwargs)
    return world, rank, local


def _reduce(x: float, op, device) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def barrier(device=None) -> None:
    """Process-group barrier (when there is one), then a device synchronisation on CUDA."""
    import torch
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)


def shard_by_weight(weights, world: int, rank: int) -> np.ndarray:
    """Indices of the items (lists, shards) that `rank` owns: contiguous runs, balanced by weight
    (e.g. removals per list). Item i goes to rank floor(world * m_i / total), m_i the midpoint of its
    weight in the running sum, so the runs are contiguous, every item has exactly one owner and the
    heaviest rank carries at most total/world + max weight."""
    w = np.asarray(weights, dtype=np.float64)
    if w.size == 0:
        return np.zeros(0, dtype=np.int64)
    if world <= 1:
        return np.arange(w.size)
    c = np.cumsum(w)
    total = c[-1]
    if total <= 0:
        owner = (np.arange(w.size) * world) // w.size
    else:
        owner = np.minimum((world * (c - 0.5 * w) / total).astype(np.int64), world - 1)
    return np.nonzero(owner == rank)[0]


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's replica: different inputs per rank, reproducible per (base, rank)."""
    return 1000 * rank + base
