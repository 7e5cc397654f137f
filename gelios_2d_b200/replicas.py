"""Host logic of the multi-GPU run: independent replicas, one process per GPU.

The step does not shard (its dt is a global minimum and surface tracking is
a serial chain), so N GPUs run N independent grids.  What crosses ranks is
timing only: every rank's device time is reduced to the maximum, and the
whole-job rate is the units all ranks processed divided by that time.  Used
by bench.py; works with any torch.distributed backend (nccl on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The maximum of ``value`` over all ranks (``value`` itself without a
    process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Units per second of the whole job: every rank processed
    ``units_per_rank`` units, the slowest took ``seconds_max``."""
    if seconds_max <= 0:
        raise ValueError("non-positive time")
    return world * units_per_rank / seconds_max
