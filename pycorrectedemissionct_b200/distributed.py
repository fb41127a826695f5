"""One process per GPU: slice sharding and the timing reductions of a multi-GPU run.

Slices are independent, so a multi-GPU solve is a partition of the slice list with no
collective on the data path; the only collectives are the barrier around a timed region and
the max-over-ranks of its duration.  Works with the ``nccl`` backend on GPUs and ``gloo`` on
CPU (tests).
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_ranks() -> tuple[int, int, int]:
    """(rank, world size, local rank) from torchrun's environment (1 process: 0, 1, 0)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def shard(total: int, rank: int, world: int) -> range:
    """Contiguous, balanced block of ``range(total)`` owned by ``rank`` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def init(backend: str, device: torch.device | None = None, timeout_s: int = 300) -> bool:
    """Initialise the process group when WORLD_SIZE > 1; returns whether one exists."""
    _, world, _ = env_ranks()
    if world <= 1:
        return False
    kw = dict(timeout=datetime.timedelta(seconds=timeout_s))
    if backend == "nccl" and device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return True


def barrier(device: torch.device | None = None) -> None:
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(value: float, device: torch.device | None = None) -> float:
    """Maximum of a per-rank scalar (e.g. a timed region's duration)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or torch.device("cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device: torch.device | None = None) -> float:
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or torch.device("cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def finalize() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
