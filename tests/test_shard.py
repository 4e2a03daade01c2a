"""The multi-GPU plumbing on CPU: world_size-2 `gloo` process groups (one process per rank, spawned), the same code the
bench runs over NCCL with one process per GPU.

* Every unit goes to exactly one rank, every rank computes the same split, and the split is balanced (LPT: no rank
  above 4/3 of the optimum).
* `combine` takes the slowest rank's seconds and the sum of the units.
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
        out[rank] = (mine, shard.combine(seconds, units))
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
    (a, (sa, ua)), (b, (sb, ub)) = results[0], results[1]
    assert sorted(a + b) == list(range(20)) and not set(a) & set(b)
    assert sa == sb == 2.0  # the slower rank's seconds
    assert ua == ub == sum(costs)


def test_a_rank_that_leaves_ends_the_others_wait_with_an_error():
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_leaving_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        results = dict(out)
    assert results == {0: "error", 1: "left"}
