"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (spawned processes,
rendezvous on 127.0.0.1) shard molecules by cost and reduce their timings
with the same helpers the GPU runs use over NCCL."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import numpy as np

from jax_examples_b200.dist import max_over_ranks, shard_by_cost, sum_over_ranks, sweep_cost, sweep_shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_by_cost(costs, rank, world)
        work = sum(costs[i] for i in mine)
        out[rank] = (mine, max_over_ranks(float(rank + 1) * 1.5), sum_over_ranks(work))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _sweep_worker(rank: int, world: int, port: int, out):
    """What bench.py's sharded sweep does before it touches a GPU: the seeded
    64-cluster sizes, this rank's share, and the reductions of its timings."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [int(x) for x in np.random.default_rng(2024).integers(1, 13, 64)]
        mine = sweep_shard(sizes, rank, world)
        cost = sum(sweep_cost(sizes[i]) for i in mine)
        out[rank] = (sizes, mine, cost, max_over_ranks(cost), sum_over_ranks(float(len(mine))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    costs = [float(n) ** 3 for n in (1, 5, 12, 3, 7, 9, 2, 11, 4, 6)]
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, _free_port(), costs, out), nprocs=2, start_method="spawn")
        res = dict(out)
    shards = [res[r][0] for r in range(2)]
    assert sorted(shards[0] + shards[1]) == list(range(len(costs)))  # each molecule exactly once
    assert shards[0] == list(range(len(shards[0])))  # contiguous
    for r in range(2):
        assert res[r][1] == pytest.approx(3.0)  # max over ranks of (rank + 1) * 1.5
        assert res[r][2] == pytest.approx(sum(costs))
    w = [sum(costs[i] for i in s) for s in shards]
    assert max(w) < 0.75 * sum(costs)  # balanced within the granularity of the units


def test_shard_by_cost_edge_cases():
    assert shard_by_cost([], 0, 2) == [] and shard_by_cost([], 1, 2) == []
    assert shard_by_cost([1.0], 0, 3) == [0] and shard_by_cost([1.0], 2, 3) == []
    assert shard_by_cost([0.0, 0.0, 0.0, 0.0], 1, 2) == [2, 3]
    parts = [shard_by_cost([1.0] * 10, r, 4) for r in range(4)]
    assert sum(parts, []) == list(range(10))
    with pytest.raises(ValueError):
        shard_by_cost([1.0], 2, 2)
    assert max_over_ranks(2.5) == 2.5  # no process group: identity


@pytest.mark.parametrize("world", [2, 3])
def test_sweep_sharded_over_gloo_ranks(world):
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_sweep_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    sizes = res[0][0]
    shards = [res[r][1] for r in range(world)]
    assert sum(shards, []) == list(range(len(sizes)))  # contiguous, in order, each molecule once
    total = sum(sweep_cost(n) for n in sizes)
    for r in range(world):
        assert res[r][3] == pytest.approx(max(res[q][2] for q in range(world)))
        assert res[r][4] == pytest.approx(len(sizes))
        # balanced to within one molecule's cost
        assert abs(res[r][2] - total / world) <= max(sweep_cost(n) for n in sizes)
