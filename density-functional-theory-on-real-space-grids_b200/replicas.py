"""Independent systems across GPUs: a cost-based partition and a host-side gather of the results.

A single system does not shard (a 65^3 grid fits one GPU many times over; a domain split would add a
7-plane halo exchange per axis per apply and FFT transposes for microseconds of work), so multi-GPU
runs are replicas. The batched workloads (a bond scan of systems on their own grids, resolution
ladders) are independent units: each rank solves its share in one batched solve, with no collective
during the solve, and rank 0 gathers the per-system scalars afterwards with one ``all_gather_object``.

The share is balanced by estimated cost, grid points x expected operator applications (the filter's
work grows with both), by the longest-processing-time rule: systems in decreasing cost, each to the
least-loaded rank (ties to the lower rank), which is deterministic on every rank and within 4/3 of the
best possible makespan.
"""

from __future__ import annotations

from typing import Any, Sequence


def system_cost(shape: Sequence[int], applications: float = 1.0) -> float:
    """Estimated work of one system: its grid points times its expected operator applications."""
    n = 1
    for s in shape:
        if int(s) <= 0:
            raise ValueError(f"grid shape {tuple(shape)} has an empty axis")
        n *= int(s)
    if not applications > 0.0:
        raise ValueError(f"expected applications must be positive, got {applications}")
    return float(n) * float(applications)


def partition_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the systems each rank solves, balanced by cost (longest processing time first).

    Every index appears exactly once; each rank's list is in increasing index order. A rank may get
    no system when there are fewer systems than ranks.
    """
    if world < 1:
        raise ValueError(f"world size must be at least 1, got {world}")
    for c in costs:
        if not c >= 0.0:
            raise ValueError(f"costs must be non-negative, got {c}")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shares[r].append(i)
        loads[r] += costs[i]
    return [sorted(s) for s in shares]


def share_loads(costs: Sequence[float], shares: Sequence[Sequence[int]]) -> list[float]:
    """The summed cost of each rank's share."""
    return [float(sum(costs[i] for i in share)) for share in shares]


def gather_by_index(local: dict[int, Any], total: int, dist=None) -> list[Any] | None:
    """Rank 0's list of all ``total`` systems' results in their original order, from each rank's
    ``{index: result}``; other ranks get None. Without a process group, ``local`` must hold them all.

    The results must be picklable host values (per-system scalars, not device tensors).
    """
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        parts = [local]
        rank = 0
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
        rank = dist.get_rank()
    if rank != 0:
        return None
    merged: dict[int, Any] = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"system {k} was solved by two ranks")
            merged[k] = v
    missing = [k for k in range(total) if k not in merged]
    if missing:
        raise ValueError(f"systems {missing} were solved by no rank")
    return [merged[k] for k in range(total)]
