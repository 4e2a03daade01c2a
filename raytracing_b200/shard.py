"""Work across GPUs: one process per GPU, the path sharded by independent units with no collective on its data.

Every unit of the path is independent: the pixels and samples of an image, the jobs of a batch, the requests of a
stream (each with its own accumulators). So N processes (one per GPU, `torch.distributed` for the plumbing) split the
units, render their share on their own GPU, and meet only to combine their timings and counts: the step time is the
slowest rank's, the work is the sum. Nothing else crosses between GPUs.

* `assign` splits units of given costs over the ranks, longest first to the least loaded rank (LPT), the same on
  every rank (a pure function of the costs), so no rank needs to hear the others' choices.
* `route` sends a stream's requests, as they arrive, each to the rank with the least outstanding work at its
  arrival: the online counterpart of `assign` for a request server on every GPU, again a pure function (of the
  arrival times and the costs), so each rank admits exactly its own requests without a message between ranks.
* `combine` reduces one rank's (seconds, units) over the process group: max of the seconds, sum of the units.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def assign(costs: Sequence[float], world: int) -> list[list[int]]:
    """The unit indices of each rank: the longest-processing-time-first split (ties by index, so every rank computes
    the same split)."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for s in shards:
        s.sort()
    return shards


def my_units(costs: Sequence[float], world: int, rank: int) -> list[int]:
    return assign(costs, world)[rank]


def route(arrivals: Sequence[float], costs: Sequence[float], world: int, rate: float) -> list[int]:
    """The rank of each request of a stream: requests taken in arrival order (equal times in index order), each sent
    to the rank whose backlog is the least when it arrives (ties to the lowest rank), where a rank's backlog is the
    cost it was sent less what it can have worked off since, at `rate` cost units a second, never below zero. With
    costs in samples (pixels x target passes) and `rate` one GPU's samples a second, a burst of large requests spreads
    over the GPUs instead of queueing behind one. Every rank computes the same list from the same arrivals, and a
    request's rank depends only on the requests that arrived before it, so routing the stream seen so far gives the
    ranks of its earlier requests unchanged: a process can route each request the moment it arrives."""
    if world < 1:
        raise ValueError("world must be at least 1")
    if len(arrivals) != len(costs):
        raise ValueError("one arrival time per cost")
    if not rate > 0:
        raise ValueError("rate must be positive")
    order = sorted(range(len(costs)), key=lambda i: (float(arrivals[i]), i))
    backlog = [0.0] * world
    now = None
    ranks = [0] * len(costs)
    for i in order:
        t = float(arrivals[i])
        if now is not None:
            worked = rate * (t - now)
            backlog = [max(0.0, b - worked) for b in backlog]
        now = t
        r = min(range(world), key=lambda k: (backlog[k], k))
        ranks[i] = r
        backlog[r] += float(costs[i])
    return ranks


def my_requests(arrivals: Sequence[float], costs: Sequence[float], world: int, rank: int, rate: float) -> list[int]:
    """The indices of the requests `route` sends to `rank`, in index order."""
    return [i for i, r in enumerate(route(arrivals, costs, world, rate)) if r == rank]


def combine(seconds: float, units: float, group=None) -> tuple[float, float]:
    """(max seconds over the ranks, sum of units over the ranks); without a process group, the rank's own."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(seconds), float(units)
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(u.item())
