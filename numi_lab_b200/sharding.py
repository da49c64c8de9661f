"""Environment sharding across GPUs (one process per GPU).

Environments are independent: a microstep has no exchange between them, so a
multi-GPU job gives each rank a contiguous environment range and runs it as
its own rollout; nothing crosses NVLink on the data path.  The only
collectives are end-of-horizon statistics: total completed env-steps
(sum) and elapsed device time (max over ranks).
"""

from __future__ import annotations

from dataclasses import dataclass


def shard_range(total_envs: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous [begin, end) environment range of `rank`."""

    if world_size <= 0 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    base, extra = divmod(total_envs, world_size)
    begin = rank * base + min(rank, extra)
    end = begin + base + (1 if rank < extra else 0)
    return begin, end


@dataclass
class HorizonStats:
    env_steps: int
    failed_env_steps: int
    device_ms: float


def reduce_stats(stats: HorizonStats, dist=None, device=None) -> HorizonStats:
    """Sums env-steps and failures and takes the max device time over ranks."""

    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return stats
    import torch

    counts = torch.tensor([stats.env_steps, stats.failed_env_steps], dtype=torch.int64, device=device)
    elapsed = torch.tensor([stats.device_ms], dtype=torch.float64, device=device)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM)
    dist.all_reduce(elapsed, op=dist.ReduceOp.MAX)
    return HorizonStats(int(counts[0].item()), int(counts[1].item()), float(elapsed[0].item()))
