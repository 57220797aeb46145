"""Multi-GPU runs of independent design points: one replica per rank, no data-path collective.

Design points (and gradient members) are independent, so N GPUs run N
replicas of a sweep; the only collective steps are a barrier around the timed
region and the maximum of the ranks' elapsed times, which is what the
whole-job throughput divides by.
"""

from __future__ import annotations


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The largest ``value`` over all ranks (every rank gets it); ``value`` itself without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds_max
