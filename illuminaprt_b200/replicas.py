"""Replica-parallel runs: one process per GPU, weak scaling.

The path's units (rays, pixels, scenes) are independent, so every rank
traces its own full copy of the workload on its own GPU and no data crosses
between ranks. The only cross-rank steps are a barrier before a timed region
and the maximum of the ranks' device times after it; the aggregate rate is
every rank's units over that maximum. Launch with torch.distributed.run (one
process per GPU); ranks read RANK / LOCAL_RANK / WORLD_SIZE from the
environment."""
from __future__ import annotations

import datetime
import os


def rank_info():
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0) -> None:
    """Joins the process group when there is more than one rank (NCCL for
    GPUs, gloo for the CPU tests); a short timeout turns a missing rank into
    an error instead of a wait."""
    import torch.distributed as dist
    world, _, _ = rank_info()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The largest of the ranks' values (each rank's timed milliseconds)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job units per second: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
