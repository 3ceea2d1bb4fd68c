"""Partitioning a batch of independent pairs over ranks (one process per GPU).

Pairs are independent, so multi-GPU runs need no exchange on the data path:
each rank solves its own contiguous shard (uniform n) or a flop-balanced set
of pairs (uneven n), and results stay on their GPU or are gathered once by the
caller.  Timing across ranks is the max over ranks.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [start, start + count) of rank `rank`; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def shard_uneven(ns, world: int, rank: int) -> np.ndarray:
    """Indices of rank `rank` for a batch of uneven sizes `ns`, balancing sum(n^3).

    Pairs are grouped by n (so each rank's pairs batch per size, as the solver
    wants) and dealt out greedily, largest cost first, to the least-loaded rank.
    Deterministic: every rank computes the same assignment.
    """
    ns = np.asarray(ns)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad shard arguments")
    order = np.lexsort((np.arange(len(ns)), -ns.astype(np.int64)))
    load = np.zeros(world)
    owner = np.empty(len(ns), dtype=np.int64)
    # deal in blocks of equal n to keep per-rank size groups contiguous
    i = 0
    while i < len(order):
        n = ns[order[i]]
        j = i
        while j < len(order) and ns[order[j]] == n:
            j += 1
        block = order[i:j]
        for start in range(0, len(block), 256):
            part = block[start:start + 256]
            r = int(np.argmin(load))
            owner[part] = r
            load[r] += float(n) ** 3 * len(part)
        i = j
    return np.sort(np.nonzero(owner == rank)[0])
