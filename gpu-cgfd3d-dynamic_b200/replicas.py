"""Replica runs across GPUs: one independent solver per rank.

The forward step keeps the whole domain on one GPU, so it has no exchange
step to distribute; N GPUs run N replicas.  These helpers give the
barrier-bracketed, max-over-ranks timing of such a run and its aggregate
rate.  Every rank takes the same collective steps in the same order.
"""
from __future__ import annotations

import datetime
import os


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """(world_size, rank, local_rank) from the torchrun environment; joins
    the process group when there is more than one rank."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return ws, rank, local


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws: int, x: float, device: str = "cuda") -> float:
    """Maximum of x over the ranks."""
    if ws <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(points: int, steps: int, ws: int, max_seconds: float) -> float:
    """Whole-job grid-point updates per second: every rank advanced its own
    replica of `points` by `steps`; the job took the slowest rank's time."""
    return points * steps * ws / max_seconds


def finish(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
