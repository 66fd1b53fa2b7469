"""Multi-rank plumbing for running independent strings on several GPUs.

The solver path has no collective: every rank owns a whole string (replicas
only).  Ranks only meet at barriers around the timed region and to combine
their device times (max over ranks) into one whole-job throughput.
"""
from __future__ import annotations

import datetime
import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend: str, device=None, timeout_s: float = 600.0) -> None:
    import torch.distributed as dist
    kw = {}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, world: int, device: str = "cpu") -> float:
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(steps_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job steps per second: the work of every rank over the slowest rank's time."""
    return world * steps_per_rank / (max_ms / 1e3)


def finalize(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
