"""Replica orchestration of the codec over ranks (one process per GPU).

The compress/decompress path has no exchange step: streams, bricks and
components are independent (own tables, own headers).  Two ways to use N
ranks, both without a collective on the data path:

* replicas: every rank codes its own volumes (weak scaling; ranks draw
  distinct inputs from their rank);
* partition: one set of bricks is split across ranks by byte size (each
  brick, largest first, to the rank with the fewest bytes so far), and the
  compressed sizes (or streams) are gathered on the host afterwards.

In both, the job's step time is the maximum over ranks of each rank's
device-timed step.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple


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


def partition_by_bytes(sizes_bytes: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the bricks each rank codes: bricks in decreasing size (ties
    by index), each to the rank holding the fewest bytes so far (ties to the
    lower rank).  Every brick goes to exactly one rank; the largest and
    smallest rank loads differ by at most the largest brick."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes_bytes)), key=lambda i: (-int(sizes_bytes[i]), i))
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes_bytes[i])
    return [sorted(p) for p in parts]


def gather_on_host(local: Dict[int, object], dist=None) -> Dict[int, object]:
    """Host-side gather of per-brick results (e.g. compressed sizes or
    streams) keyed by brick index: every rank gets the union."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    out: Dict[int, object] = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise ValueError(f"brick {k} coded on two ranks")
            out[k] = v
    return out
