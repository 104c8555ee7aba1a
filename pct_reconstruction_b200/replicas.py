"""Independent reconstructions on several GPUs (one process per GPU).

The DROP path has no profitable split inside a block at the reference's block sizes: splitting
histories across GPUs would need an all-reduce of the {x_update, S} accumulator (10 MB for a
200x200x32 grid) after every one of the ~800 blocks of an iteration.  Multi-GPU runs are
therefore replicas: each rank reconstructs its own scan (its own seed / data), nothing crosses
ranks on the data path, and only the timing is combined -- the slowest rank's time, taken on the
device and reduced with MAX, over the histories of all ranks (weak scaling).
"""
from __future__ import annotations

import os


def world() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment (single process: 0, 0, 1)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def replica_seed(base: int, rank: int) -> int:
    """Seed of the synthetic scan a rank reconstructs (distinct per rank)."""
    return base + 1000003 * rank


def max_over_ranks(value: float, device=None) -> float:
    """Largest value over all ranks (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(histories_per_rank: int, ms_per_step_local: float, device=None) -> tuple[float, float]:
    """(whole-job histories/s, slowest rank's ms per step) for replicas of equal size."""
    import torch.distributed as dist
    n_ranks = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    ms = max_over_ranks(ms_per_step_local, device)
    return histories_per_rank * n_ranks / (ms / 1000.0), ms
