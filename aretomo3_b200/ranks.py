"""Rank plumbing for multi-GPU runs of the reconstruction path.

Every y-slice is independent, so N GPUs take N shares of the work with no
exchange on the data path: either N series (replicas, weak scaling, what
bench.py --gpus N runs) or N y-slabs of one series (rows_of_rank).  The only
collectives are the barrier around timed regions and the max over ranks of a
time (torch.distributed: NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def distributed() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    if distributed():
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, device=None) -> float:
    """The largest x over all ranks (a time: the job takes as long as its
    slowest rank).  device: where the reduction tensor lives (a CUDA device
    under NCCL, None for gloo)."""
    if not distributed():
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rows_of_rank(ny: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous y-slab [y0, y1) of rank `rank` when one series of ny rows is
    split over `world` ranks: sizes differ by at most one row, lower ranks
    take the extra rows, every row belongs to exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(ny, world)
    y0 = rank * base + min(rank, extra)
    return y0, y0 + base + (1 if rank < extra else 0)


def aggregate_rate(units_per_rank: float, steps: int, world: int, max_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time (ms), per second."""
    return units_per_rank * steps * world / (max_ms / 1e3)
