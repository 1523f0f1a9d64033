"""Multi-process plumbing for running the counter on several GPUs of a node.

The per-vertex count has no exchange step when each GPU counts its own
graphs: the batched and served workloads shard by graph, and the benchmark
runs one independent replica per GPU.  What crosses processes is only
bookkeeping: a barrier around the timed region and the max of the ranks'
device times (the job takes as long as its slowest rank).  These helpers do
exactly that over torch.distributed (NCCL on GPUs, gloo on hosts).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(rank, world size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (identity on one process)."""
    rank, size = world()
    if size == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(count: int, rank: int, size: int) -> range:
    """Contiguous block of items [begin, end) owned by `rank` of `size`."""
    per, extra = divmod(count, size)
    begin = rank * per + min(rank, extra)
    return range(begin, begin + per + (1 if rank < extra else 0))
