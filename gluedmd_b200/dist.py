"""Multi-GPU plumbing for the batched path: one process per GPU.

Walkers are independent, so they shard across ranks with no data-path
collective (weak scaling: each rank evaluates its own walkers). The
collectives are the timing reductions of the benchmark (max over ranks), the
barriers around the timed region, and the periodic bias-state sync between
walker groups (``sync_bias_state``). NCCL on GPUs, gloo for the CPU tests.
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


def sync_bias_state(blob, force, baselines=None, group=None):
    """Cross-rank bias sync of one walker group per rank (the CPU-mediated merge of
    python/MultiGPUManager.py:1076-1113, with ranks in place of device groups).

    Every rank passes its group's ``getBiasState()`` blob; the blobs are gathered
    on every rank (``all_gather_object``, rank order) and each rank computes the
    same incremental additive merge, so all ranks return the identical merged
    blob, to load with ``setBiasState``, and the baselines to pass back at the
    next sync. Without an initialized process group the blob is returned as is.
    Every rank must call this at the same step.
    """
    from .merger import BiasStateMerger
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return bytes(blob), [BiasStateMerger._parse(bytes(blob), force)]
    world = dist.get_world_size(group)
    blobs = [None] * world
    dist.all_gather_object(blobs, bytes(blob), group=group)
    return BiasStateMerger.merge_additive_incremental(blobs, force, baselines)
