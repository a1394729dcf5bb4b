"""Multi-GPU replicas of the plain sort: each LSD pass is a global permutation, so the plain
sort does not shard without an exchange step; N ranks run N independent sorts (weak
scaling).  These helpers combine the ranks' timings: the job takes as long as its slowest
rank, and the job's throughput counts every rank's keys."""
from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (identity when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_gkeys(keys_per_rank_per_step: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job throughput in Gkeys/s: all ranks' keys over the slowest rank's time."""
    return keys_per_rank_per_step * steps * world / (max_ms / 1e3) / 1e9
