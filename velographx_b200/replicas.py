"""Host logic of multi-GPU runs: independent replicas, one process per GPU.

The dynamic-BFS path has no exchange step: every rank holds its own copy of
the graph and applies the same batches (or its own share of BFS roots), and
only the timing is combined.  ``torch.distributed`` is the plumbing (NCCL on
GPUs, gloo on CPU for the tests).
"""
from __future__ import annotations

import datetime
import os


def init(backend: str, timeout_s: float = 120.0):
    """Joins the process group of a torchrun launch (RANK, WORLD_SIZE,
    MASTER_ADDR/PORT in the environment); returns (rank, world)."""
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist.get_rank(), dist.get_world_size()


def max_over_ranks(x: float, device: str = "cpu") -> float:
    """The largest of every rank's x (the whole job ends when its slowest rank
    does); x itself when no process group is running."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank: int, world: int):
    """Rank `rank`'s share of `items` (every item in exactly one share, sizes
    differing by at most one): the BFS roots of a multi-root run split across
    replicas."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return items[rank::world]


def env_rank_world(default_world: int = 1):
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", default_world))
