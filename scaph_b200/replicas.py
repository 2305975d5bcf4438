"""Replica plumbing for multi-GPU runs (one process per GPU).

The BFS path has no data exchange: the graph is replicated and each rank
runs its own sources.  The only collective is the timing reduction (the
slowest rank's device time); the data path never touches a collective.
"""
from __future__ import annotations


def rank_sources(sources: list[int], rank: int, steps: int) -> list[int]:
    """The `steps` sources rank `rank` runs: a rank-dependent rotation of the
    shared seeded source list, so replicas do different traversals."""
    n = len(sources)
    return [sources[(rank * 7 + i) % n] for i in range(steps)]


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Maximum of `value` over all ranks (identity when world == 1)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gteps(world: int, steps: int, edges: int, ms_max: float) -> float:
    """Whole-job GTEPS: every rank traverses `steps` times `edges` edges;
    the job takes as long as its slowest rank."""
    return world * steps * edges / (ms_max / 1e3) / 1e9
