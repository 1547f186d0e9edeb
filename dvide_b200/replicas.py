"""Replica placement for more than one GPU.

The contact step does not shard inside a scene (every Schur product couples
contacts through shared bodies), so N GPUs run replicas: independent scenes
are placed on ranks by a greedy longest-processing-time bin packing of their
estimated cost (bodies + 3 x contacts), with no collective on the data path.
After a timed region the ranks combine their counts once: contacts summed,
times maximised (the job is as slow as its slowest rank)."""
from __future__ import annotations

import heapq


def scene_cost(nb: int, nc: int = 0) -> float:
    """Estimated per-step cost of a scene (bodies + 3 x contacts; 4 x bodies
    stands in for the contacts of a scene that has not been stepped)."""
    return float(nb) + 3.0 * float(nc if nc else 4 * nb)


def partition_by_cost(costs, nparts: int):
    """Greedy LPT: scenes by decreasing cost, each to the least-loaded rank.
    Deterministic (ties by scene index, then rank).  Returns one sorted index
    list per rank."""
    if nparts <= 0:
        raise ValueError("nparts must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(nparts)]
    heapq.heapify(heap)
    parts = [[] for _ in range(nparts)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def combine_timed_region(dist, contacts: float, seconds: float, device=None):
    """(sum of contacts over ranks, max of seconds over ranks); plain values
    when dist is None (one rank)."""
    if dist is None:
        return float(contacts), float(seconds)
    import torch
    t = torch.tensor([float(contacts), float(seconds)], dtype=torch.float64, device=device)
    s = t.clone()
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    m = t.clone()
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(s[0].item()), float(m[1].item())
