"""Partition of an ensemble's members over GPU ranks (the multi-GPU path's host logic).

Members are independent domains, so a multi-GPU run gives each rank a disjoint set of whole
members and needs no collective inside a step.  To split one fixed ensemble (strong scaling), the
members are assigned greedily by cost, largest first, each to the rank with the least cost so far
(longest-processing-time order).  The cost of a member is its interior cells times the physical
steps it takes; every member of a batch takes the same steps, so cells alone order them.
"""
from __future__ import annotations


def partition_by_cost(costs: list, world: int) -> list:
    """Member indices per rank: disjoint, together all of them, each rank's list ascending.

    Ties are broken by index (members) and by rank number (ranks), so every rank computes the same
    partition from the same costs without exchanging anything."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += costs[i]
        shards[r].append(i)
    return [sorted(s) for s in shards]
