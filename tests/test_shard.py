"""The multi-GPU plumbing on CPU: world_size-2 `gloo` process groups (one process per rank, spawned), the same code the
bench runs over NCCL with one process per GPU.

* Every unit goes to exactly one rank, every rank computes the same split, and the split is balanced (LPT: no rank
  above 4/3 of the optimum).
* `combine` takes the slowest rank's seconds and the sum of the units.
* `route` sends each request of a stream to exactly one rank, the same on every rank (two gloo ranks computing their
  own requests apart), the least-backlogged one at its arrival: the rule restated event by event gives the same
  ranks, a burst spreads over the ranks, and requests spaced wider than their work stay on the first.
* A rank that fails raises on its own and the group's timeout ends the others' wait: no rank hangs.
"""
import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from raytracing_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.my_units(costs, world, rank)
        seconds = 1.0 + rank  # the slower rank decides the step
        units = sum(costs[i] for i in mine)
        arrivals = [0.05 * i for i in range(len(costs))]
        requests = shard.my_requests(arrivals, costs, world, rank, rate=40.0)
        out[rank] = (mine, shard.combine(seconds, units), requests)
    finally:
        dist.destroy_process_group()


def _leaving_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        if rank == 1:
            out[rank] = "left"  # this rank leaves between steps, without taking part in the combine
            return
        try:
            shard.combine(1.0, 1.0)
            out[rank] = "combined"
        except RuntimeError:
            out[rank] = "error"  # the group's timeout (or the closed peer) ends the wait with an error
    finally:
        dist.destroy_process_group()


def test_assign_is_complete_disjoint_and_balanced():
    costs = [float((i * 37) % 101 + 1) for i in range(64)]
    for world in (1, 2, 3, 8):
        shards = shard.assign(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) <= 4 / 3 * max(sum(costs) / world, max(costs)) + 1e-9
        assert shards == shard.assign(costs, world)  # a pure function: every rank computes the same split
    with pytest.raises(ValueError):
        shard.assign(costs, 0)


def _brute_route(arrivals, costs, world, rate):
    """The same rule restated event by event: every request's rank from the backlogs of all requests before it."""
    order = sorted(range(len(costs)), key=lambda i: (arrivals[i], i))
    sent = []  # (rank, arrival, cost) in arrival order
    ranks = [None] * len(costs)
    for i in order:
        backlog = []
        for k in range(world):
            b, last = 0.0, None
            for r, t, c in sent:
                if last is not None:
                    b = max(0.0, b - rate * (t - last))
                last = t
                if r == k:
                    b += c
            if last is not None:
                b = max(0.0, b - rate * (arrivals[i] - last))
            backlog.append(b)
        best = min(range(world), key=lambda k: (backlog[k], k))
        ranks[i] = best
        sent.append((best, arrivals[i], costs[i]))
    return ranks


def test_route_spreads_a_burst_and_matches_its_rule():
    import random

    gen = random.Random(3)
    for world in (1, 2, 3, 8):
        arrivals = sorted(gen.uniform(0, 2) for _ in range(60))
        arrivals[10] = arrivals[11]  # equal arrival times go in index order
        costs = [gen.choice([1.0, 4.0, 16.0, 64.0]) for _ in range(60)]
        ranks = shard.route(arrivals, costs, world, rate=20.0)
        assert all(0 <= r < world for r in ranks)
        assert ranks == shard.route(arrivals, costs, world, rate=20.0)  # the same on every rank
        assert ranks == _brute_route(arrivals, costs, world, 20.0)
        mine = [shard.my_requests(arrivals, costs, world, k, 20.0) for k in range(world)]
        assert sorted(i for m in mine for i in m) == list(range(60))
        for cut in (1, 17, 59):  # online: the stream seen so far routes its requests as the whole stream does
            assert shard.route(arrivals[:cut], costs[:cut], world, rate=20.0) == ranks[:cut]
    # a burst at one instant goes round the ranks; requests spaced wider than their work all go to the first
    assert shard.route([0.0] * 6, [5.0] * 6, 3, rate=1.0) == [0, 1, 2, 0, 1, 2]
    assert shard.route([0.0, 10.0, 20.0], [5.0] * 3, 3, rate=1.0) == [0, 0, 0]
    # the large request's rank is passed over while its backlog lasts
    assert shard.route([0.0, 0.1, 0.2, 0.3], [100.0, 1.0, 1.0, 1.0], 2, rate=1.0) == [0, 1, 1, 1]
    for bad in ((0, 1.0), (2, 0.0)):
        with pytest.raises(ValueError):
            shard.route([0.0], [1.0], bad[0], rate=bad[1])
    with pytest.raises(ValueError):
        shard.route([0.0, 1.0], [1.0], 2, rate=1.0)


def test_combine_without_a_group_is_the_rank_itself():
    assert shard.combine(2.5, 7) == (2.5, 7.0)


def test_two_gloo_ranks_split_and_combine():
    costs = [float(i % 7 + 1) for i in range(20)]
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_worker, args=(world, _free_port(), costs, out), nprocs=world, start_method="spawn")
        results = dict(out)
    assert sorted(results) == [0, 1]
    (a, (sa, ua), ra), (b, (sb, ub), rb) = results[0], results[1]
    assert sorted(a + b) == list(range(20)) and not set(a) & set(b)
    # each rank's own requests of the stream, computed apart: together every request once, as route() splits them
    assert sorted(ra + rb) == list(range(20)) and ra and rb
    ranks = shard.route([0.05 * i for i in range(20)], costs, world, rate=40.0)
    assert ra == [i for i in range(20) if ranks[i] == 0] and rb == [i for i in range(20) if ranks[i] == 1]
    assert sa == sb == 2.0  # the slower rank's seconds
    assert ua == ub == sum(costs)


def test_a_rank_that_leaves_ends_the_others_wait_with_an_error():
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_leaving_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        results = dict(out)
    assert results == {0: "error", 1: "left"}
