"""Multi-GPU plumbing for the batched path: one process per GPU.

Walkers are independent, so they shard across ranks with no data-path
collective (weak scaling: each rank evaluates its own walkers). The only
collectives are the timing reductions of the benchmark (max over ranks) and
the barriers around the timed region. NCCL on GPUs, gloo for the CPU tests.
"""
from __future__ import annotations

import datetime
import os


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items, rank, world):
    """Contiguous block partition of n_items over world ranks: (start, stop)."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def init(backend, timeout_s=120):
    import torch.distributed as dist
    if dist.is_available() and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x, device="cpu"):
    """Max of a float over all ranks (identity without an initialized group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, device="cpu"):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
