"""Set-level sharding of the batched and served forms over the GPUs of one node.

Independent particle sets (and requests) need no exchange: each rank solves its own
share and only the per-rank timings and counts are reduced.  Shares are formed by the
longest-processing-time rule on the sets' particle counts (the work of a solve grows
with its particles), so the slowest rank -- which sets the job's time -- carries as
little as the packing allows.  Host-only; the reductions use whatever process group
torch.distributed was initialised with (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import Sequence


def pack_sets(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the sets each rank solves: largest set first onto the least-loaded
    rank (ties to the lower rank).  Every set lands on exactly one rank; each rank's
    list is in ascending set order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shares: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(s) for s in shares]


def pack_requests(reqs: Sequence[dict], world: int) -> list[int]:
    """Rank of each request of a served stream: new sets packed by particle count in
    arrival order (onto the rank with the least particles so far), continuations on the
    rank that holds their set (they need its device-resident state)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    rank = [0] * len(reqs)
    for k, e in enumerate(reqs):
        if e["kind"] == "new":
            r = min(range(world), key=lambda q: (load[q], q))
            load[r] += int(e["n"])
            rank[k] = r
        else:
            rank[k] = rank[e["of"]]
    return rank


def imbalance(sizes: Sequence[int], shares: Sequence[Sequence[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect)."""
    loads = [sum(int(sizes[k]) for k in s) for s in shares]
    mean = sum(loads) / max(1, len(loads))
    return max(loads) / mean if mean > 0 else 1.0


def reduce_scalar(dist, value: float, op: str = "max", device=None) -> float:
    """All-reduce of one float over the process group (max or sum); the value itself
    when dist is None."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def gather_floats(dist, values: Sequence[float], world: int) -> list[float]:
    """Every rank's list of floats, concatenated in rank order, on every rank."""
    if dist is None:
        return list(values)
    out = [None] * world
    dist.all_gather_object(out, [float(v) for v in values])
    return [v for part in out for v in part]
