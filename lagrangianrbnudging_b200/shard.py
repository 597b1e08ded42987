"""Splitting independent units over GPUs (one process per GPU, no data-path
collective).

The configurations with more than one unit have independent units: the
members of an ensemble, the nudging coefficients of a twin-experiment sweep,
the seeded directions of a finite-difference check.  Each rank runs its own
share on its own GPU; only the final results (and the slowest rank's time)
cross ranks, once, after the work.  The reference has no counterpart: its
MPI ranks share one domain.
"""
from __future__ import annotations

from typing import Sequence


def lpt(costs: Sequence[float], nparts: int) -> list[list[int]]:
    """Longest processing time first: units in decreasing cost (ties by index)
    go one by one to the part with the least load so far (ties by the lower
    part).  Every unit lands in exactly one part; each part's unit list is in
    increasing index order.  The largest load is at most 4/3 of the optimum
    (Graham's bound)."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    load = [0.0] * nparts
    parts: list[list[int]] = [[] for _ in range(nparts)]
    for i in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        p = min(range(nparts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += float(costs[i])
    return [sorted(p) for p in parts]


def my_units(costs: Sequence[float], rank: int, world: int) -> list[int]:
    """the units of `rank` out of `world` ranks (every rank computes the same
    split from the same costs)"""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return lpt(costs, world)[rank]


def gather(dist, obj):
    """every rank's `obj`, in rank order (one all-gather of Python objects);
    [obj] without a process group"""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
