"""Replica and ensemble bookkeeping for one process per GPU (``bench.py --gpus N``).

One IBPM simulation does not shard: its multi-domain solve is global per
level and the levels are serially dependent.  N GPUs therefore run N
independent replicas; a job's throughput is the units every rank processed
divided by the slowest rank's time.  An ensemble of independent simulations
shards by member instead: rank r advances members r, r + N, r + 2N, ... with
no exchange while they run, and one all-gather collects the members' force
histories at the end.  These helpers hold that arithmetic so that it runs the
same way over NCCL (CUDA tensors) and over gloo (CPU tensors, as the
multi-process tests use it).
"""
from __future__ import annotations


def world():
    """(world size, rank, local rank) from the torchrun environment."""
    import os
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (the
    value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world_size: int, steps: int, units_per_step: int, max_ms: float) -> float:
    """Units per second of the whole job: every rank advanced `steps` steps of
    `units_per_step` units; the job took as long as its slowest rank."""
    if max_ms <= 0:
        raise ValueError("the timed region must have a positive duration")
    return world_size * steps * units_per_step / (max_ms / 1000.0)


def shard(units: int, world_size: int, rank: int) -> list:
    """The members (of `units`) that rank `rank` of `world_size` advances: every
    world_size-th one from `rank`, so uneven member sizes spread over the ranks."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank outside the world")
    return list(range(rank, units, world_size))


def gather_histories(local, units: int, device=None):
    """All-gather per-member histories: `local` is this rank's (len(shard), ...) array in
    shard order; every rank gets the (units, ...) array in member order."""
    import numpy as np
    import torch
    import torch.distributed as dist
    local = np.asarray(local, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    ws, rank = dist.get_world_size(), dist.get_rank()
    per = -(-units // ws)                                   # the most members a rank holds
    buf = np.zeros((per,) + local.shape[1:])
    buf[: local.shape[0]] = local
    t = torch.as_tensor(buf, device=device)
    parts = [torch.empty_like(t) for _ in range(ws)]
    dist.all_gather(parts, t)
    out = np.empty((units,) + local.shape[1:])
    for r, part in enumerate(parts):
        mine = shard(units, ws, r)
        out[mine] = part.cpu().numpy()[: len(mine)]
    return out
