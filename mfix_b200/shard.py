"""Sharding of independent systems across ranks (one process per GPU).

The path has no data exchange between systems: a batch of independent
systems (the SIMPLE loop's per-phase / per-direction solves,
model/solve_vel_star.f:315-331) is split across ranks and each rank solves
its share with no collective on the data path.  Only host-side bookkeeping
crosses ranks: the maximum of the per-rank device times and the totals.
"""
from __future__ import annotations


def assign(cells: list[int], world: int) -> list[list[int]]:
    """Greedy longest-first assignment of systems to ranks by cell count (a
    solve's traffic is proportional to its cells).  Returns, per rank, the
    system indices in ascending order.  Every system goes to exactly one rank,
    and the most loaded rank holds at most the mean load plus one system."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(cells)), key=lambda q: (-cells[q], q))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(q)
        load[r] += cells[q]
    return [sorted(v) for v in out]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (the
    value itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
