"""Multi-GPU runs of independent design points: one sweep partitioned across ranks, no data-path collective.

Design points (and gradient members) are independent, so N GPUs split one
sweep of N times the per-GPU point count: rank r marches points r, r + N,
r + 2N, ... as its own batch (src/sweep.py:416-436 runs the same points one
after another, or over a process pool).  The only collective steps are a
barrier around the timed region, the maximum of the ranks' elapsed times
(what the whole-job throughput divides by) and a host-side sum of the
ranks' converged counts and outcome tallies.
"""

from __future__ import annotations


def partition(items, rank: int, world: int) -> list:
    """Rank ``rank``'s share of ``items``: every ``world``-th item from position ``rank`` (disjoint, covering)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in a world of {world}")
    return list(items)[rank::world]


def _reduce(values, dist, device, op):
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op(dist))
    return [float(v) for v in t.cpu().tolist()]


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The largest ``value`` over all ranks (every rank gets it); ``value`` itself without a process group."""
    return _reduce([value], dist, device, lambda d: d.ReduceOp.MAX)[0]


def sum_over_ranks(values, dist=None, device="cpu") -> list:
    """Element-wise sums of a short list of numbers over all ranks (every rank gets them)."""
    return _reduce(values, dist, device, lambda d: d.ReduceOp.SUM)


def whole_job_rate(units_all_ranks: float, seconds_max: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return units_all_ranks / seconds_max
