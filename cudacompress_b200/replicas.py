"""Replica orchestration of the codec over ranks (one process per GPU).

The compress/decompress path has no exchange step: every rank codes its own
volumes (weak scaling, no data crosses ranks).  The only cross-rank steps are
host-side: ranks draw distinct inputs from their rank, and the job's step time
is the maximum over ranks of each rank's device-timed step, so the job's
throughput is (ranks x bytes per rank-step) / that maximum.
"""
from __future__ import annotations

from typing import Sequence, Tuple


def rank_seeds(seeds: Sequence[int], rank: int) -> Tuple[int, ...]:
    """Input seeds of a rank: distinct for every rank, rank 0 keeps `seeds`."""
    return tuple(int(s) + 100 * int(rank) for s in seeds)


def max_over_ranks(values: Sequence[float], dist=None, device=None) -> list:
    """Element-wise maximum of `values` over all ranks (identity without a
    process group).  Every rank must call it with the same length."""
    vals = [float(v) for v in values]
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    import torch
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_gbs(world: int, bytes_per_rank_step: int, step_ms: float) -> float:
    """Whole-job throughput in GB/s: all ranks' bytes over the slowest rank's step."""
    if step_ms <= 0:
        raise ValueError("step time must be positive")
    return world * bytes_per_rank_step / (step_ms / 1e3) / 1e9
