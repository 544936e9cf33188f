"""Replica parallelism: one independent domain per rank (torch.distributed).

The LBM step has no exchange between independent domains (ensemble members or
replicas), so ranks share nothing on the data path.  The process group is used
only for the barrier around timed regions and the max over ranks of elapsed
time.  Works with the nccl backend on GPUs and with gloo on CPU.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def init(backend: str, timeout_s: float = 120.0, device=None):
    """Initialise the default process group from the torchrun environment (127.0.0.1 rendezvous)."""
    kw = {}
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def max_over_ranks(value: float, device="cpu") -> float:
    """Max of a scalar over all ranks (every rank gets the result)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Seed of the replica a rank advances (distinct per rank, reproducible)."""
    return int(base) + 1000003 * int(rank)


def shard(n_items: int, world: int, rank: int):
    """Round-robin assignment of items (ensemble members) to ranks: every item exactly once."""
    return list(range(rank, n_items, world))
