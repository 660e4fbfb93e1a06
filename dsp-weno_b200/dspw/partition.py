"""Partition of a batch of independent problems over ranks (one process per GPU).

Problems of a batch never exchange data, so a multi-GPU run needs no
data-path collective: every rank advances its own share in one handle, and
the only communication is the barrier and the max-over-ranks of the device
time.  The share is balanced by cell count (the work of one step is
proportional to the cells a problem holds), largest problem first onto the
least-loaded rank, ties to the lower rank, so every rank computes the same
assignment from the problem list alone.
"""
from __future__ import annotations

import heapq


def partition(cells, world: int):
    """Indices of the problems of each rank: a list of ``world`` sorted index
    lists covering ``range(len(cells))`` exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(cells[i]), r))
    return [sorted(s) for s in out]


def loads(cells, parts):
    return [sum(int(cells[i]) for i in p) for p in parts]


def imbalance(cells, parts) -> float:
    """max rank load / mean rank load (1.0 is perfect balance)."""
    ld = loads(cells, parts)
    mean = sum(ld) / len(ld)
    return max(ld) / mean if mean > 0 else 1.0
