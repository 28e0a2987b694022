"""Multi-GPU replicas of the splatting path (one process per GPU).

Frames are independent units (one camera each), so N GPUs render disjoint
subsets of the orbit with no exchange on the data path; the only collective
is the end-of-run reduction of the timing (max over ranks), which
torch.distributed performs over NCCL on GPUs or gloo on CPUs.
"""
from __future__ import annotations


def frame_index(rank: int, world: int, step: int, frames: int) -> int:
    """Camera index rendered by `rank` at global step `step` (round robin)."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    return (rank + step * world) % frames


def frames_for_rank(rank: int, world: int, first_step: int, steps: int, frames: int) -> list[int]:
    return [frame_index(rank, world, first_step + i, frames) for i in range(steps)]


def reduce_max(value: float, dist=None, device=None) -> float:
    """Max of `value` over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, seconds_max: float) -> float:
    """Units of all ranks divided by the slowest rank's time."""
    return world * units_per_rank / seconds_max
