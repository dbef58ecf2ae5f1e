"""Running the element loop as independent replicas, one process per GPU.

The loop shards by element with no exchange inside an evaluation, so N GPUs
run N independent meshes (weak scaling): no collective touches the data
path. The process group only lines the ranks up around the timed region and
takes the slowest rank's time, so that the whole-job rate is the units all
ranks processed divided by the time of the slowest.
"""
from __future__ import annotations

import os
from datetime import timedelta


def rank_env() -> tuple:
    """(rank, world size, local rank) from torchrun's environment."""

    def get(name, default):
        try:
            return int(os.environ.get(name, default))
        except ValueError:
            return default

    return get("RANK", 0), get("WORLD_SIZE", 1), get("LOCAL_RANK", 0)


def init(world: int, backend: str, device=None, timeout_s: float = 600.0) -> bool:
    """Join the process group when there is more than one rank; the short
    timeout makes ranks that wait for a missing peer fail instead of hang."""
    if world <= 1:
        return False
    import torch.distributed as dist

    kw = {"device_id": device} if device is not None and backend == "nccl" else {}
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return True


def replica_seed(base: int, rank: int) -> int:
    """Each replica evaluates its own mesh of the same construction."""
    return base + rank


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The largest `value` of all ranks (every rank gets it)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds


def finish(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
