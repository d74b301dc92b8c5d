"""Whole cases across GPUs: one process per GPU, each running its share of a
case list as one batch, with no data exchange between ranks.

The reference runs one case on many MPI ranks, a block or more per rank
(`m2node`, sub_init_readbcinfo.f90); here all blocks of a case stay on one
GPU, and several GPUs share a list of independent cases instead.  The split
is longest-processing-time-first on the cases' node counts (each case goes,
largest first, to the rank with the least work so far; ties go to the lower
rank and the lower case index), a pure function of the list, so every rank
computes the same assignment without talking to the others.  Its largest
rank load is at most 4/3 of the optimum (Graham, SIAM J. Appl. Math. 17,
1969).  Results come back to rank 0 by `gather`, in case order.
"""
from __future__ import annotations

from typing import Any, Callable, Dict, List, Optional, Sequence


def assign(costs: Sequence[int], world: int) -> List[List[int]]:
    """Case indices per rank (each list in ascending case order)."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda c: (-int(costs[c]), c)):
        r = min(range(world), key=lambda x: (load[x], x))
        out[r].append(i)
        load[r] += int(costs[i])
    return [sorted(x) for x in out]


def share(cases: Sequence[Any], rank: int, world: int, cost: Callable[[Any], int] = lambda c: c.nodes):
    """(indices, cases) of this rank's share."""
    idx = assign([cost(c) for c in cases], world)[rank]
    return idx, [cases[i] for i in idx]


def gather(results: Dict[int, Any], dist=None) -> Optional[Dict[int, Any]]:
    """Per-case results of every rank on rank 0 (others get None); without a
    process group, the local results."""
    if dist is None:
        return dict(sorted(results.items()))
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(results, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: Dict[int, Any] = {}
    for p in parts:
        merged.update(p)
    return dict(sorted(merged.items()))
