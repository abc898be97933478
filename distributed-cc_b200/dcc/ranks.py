"""Timing across the ranks of one job (one process per GPU, launched by torchrun).

The triples path does not shard here (one GPU holds all canonical blocks), so a job of N
ranks runs N independent replicas of the same iteration: there is no collective in the data
path.  The only cross-rank operations are the barrier around the timed region and the
maximum of the per-rank times, since the job's time is that of its slowest rank."""
from __future__ import annotations

import torch


def world():
    """(rank, world size) of the default process group, (0, 1) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def barrier(device=None):
    """Every rank reaches this point (and, with a CUDA device, its queued work has finished)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(value, device="cpu"):
    """The largest of the ranks' values (every rank gets it).  `device` is where the one-element
    tensor of the all-reduce lives: "cuda" for NCCL, "cpu" for gloo."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_seconds_per_iteration(max_ms, steps, world_size):
    """Whole-job seconds per iteration for `world_size` replicas that each ran `steps` iterations
    in `max_ms` (the slowest rank's time): the job completes world_size iterations per step time."""
    if steps <= 0 or world_size <= 0:
        raise ValueError("steps and world_size must be positive")
    return max_ms / steps / 1e3 / world_size
