"""Event sharding across GPUs: one event list, split by sorted-multiplicity round-robin.

Events and primary vertices are independent (the reference loops over them with no shared state,
Tracker.cxx:251-262), so a multi-GPU run splits one list of events across ranks with no collective
on the data path. The work of an event grows about as the square of its multiplicity (the tracklet
and cell candidates of a bin window), so the events are ordered by that cost, largest first, and
dealt to the ranks in a snake: 0, 1, ..., W-1, W-1, ..., 1, 0, 0, 1, ... Every rank then holds
events of every size, and the largest events do not pile up on the first ranks.
"""
from __future__ import annotations

import numpy as np


def event_cost(multiplicity) -> np.ndarray:
    """The relative cost of events of the given multiplicities (tracks or clusters): N^2."""
    m = np.asarray(multiplicity, np.float64)
    return m * m


def partition(costs, world: int) -> list:
    """Indices of the events of each of `world` ranks: sorted by cost, largest first (ties by
    index), dealt in a snake. Each rank's list is in ascending event order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, np.float64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    shards = [[] for _ in range(world)]
    for k, e in enumerate(order):
        lap, pos = divmod(k, world)
        shards[pos if lap % 2 == 0 else world - 1 - pos].append(int(e))
    return [sorted(s) for s in shards]


def imbalance(costs, shards) -> float:
    """Largest rank cost over the mean rank cost, minus one (0: perfectly even)."""
    costs = np.asarray(costs, np.float64)
    loads = np.array([costs[s].sum() for s in shards])
    return float(loads.max() / loads.mean() - 1.0) if loads.mean() > 0 else 0.0
