"""Sharding independent state points across ranks (one process per GPU).

The state points of an isotherm (or of several) are independent converge! problems: no
data crosses ranks while they converge.  Ranks take disjoint subsets balanced by an
estimate of their cost (longest processing time first), converge them as one batch each,
and rank 0 gathers (γ, adsorption, status, ρ) of every state point afterwards -- a host
gather outside the timed region, the only communication.

The cost of a state point is its evaluation count times the cost of one evaluation; the
count is not known before converging, so the estimate is the per-evaluation cost of the
1D engine, which grows with the square of the grid size (the circulant convolutions).
"""
import heapq

import numpy as np


def estimated_cost(ngrid, nc=1):
    """Per-evaluation cost estimate of a 1D system of ``ngrid`` points and ``nc`` components."""
    return float(nc) * float(ngrid) ** 2


def lpt_partition(costs, nranks):
    """Longest-processing-time-first assignment of items with ``costs`` to ``nranks`` ranks.

    Returns a list of index lists, one per rank, each sorted ascending (the batch order).
    Items go, largest first, to the rank with the smallest load so far (ties: lowest rank)."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    parts = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def gather_results(dist, rank, world, indices, records, total):
    """Gather per-state-point records (any picklable object) from every rank to rank 0.

    ``indices`` are this rank's state-point indices, ``records`` the matching results.
    Rank 0 returns the list of ``total`` records in global order; other ranks return None."""
    mine = list(zip(indices, records))
    if world == 1 or dist is None:
        out = [None] * total
        for i, r in mine:
            out[i] = r
        return out
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * total
    for part in gathered:
        for i, r in part:
            if out[i] is not None:
                raise RuntimeError(f"state point {i} converged on two ranks")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"state points {missing} were not converged by any rank")
    return out


def balance(parts, costs):
    """Largest rank load over the mean load (1 = perfect balance)."""
    loads = np.array([sum(costs[i] for i in p) for p in parts])
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0
