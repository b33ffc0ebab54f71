"""Multi-process plumbing for replicas on several GPUs (one process per GPU).

The two-electron path shards without a data exchange when the units are
independent molecules or geometries: each rank takes a contiguous,
cost-balanced share of the molecules (``shard_by_cost``) and runs them as
its own batch; the only collectives are the timing reductions of the
benchmark (``max_over_ranks``) and barriers.  Sharding one molecule's quartet
list over ranks would add one all-reduce of J/K per build; that form is not
built.  Works with the ``nccl`` backend on GPUs and with ``gloo`` on CPU
(the tests).
"""

from __future__ import annotations

import os
from typing import List, Sequence, Tuple

import torch
import torch.distributed as dist


def env_ranks() -> Tuple[int, int, int]:
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_by_cost(costs: Sequence[float], rank: int, world: int) -> List[int]:
    """Indices of the contiguous share of units for ``rank``: the split points
    are where the running cost crosses k/world of the total, so every rank
    gets about the same cost and every unit goes to exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    total = float(sum(costs))
    if total <= 0.0:
        n = len(costs)
        return list(range(rank * n // world, (rank + 1) * n // world))
    bounds = [0]
    acc = 0.0
    k = 1
    for i, c in enumerate(costs):
        acc += float(c)
        while k < world and acc >= total * k / world:
            bounds.append(i + 1)
            k += 1
    while len(bounds) < world:
        bounds.append(len(costs))
    bounds.append(len(costs))
    return list(range(bounds[rank], bounds[rank + 1]))


def sweep_cost(n_waters: int) -> float:
    """Estimated cost of one water cluster's energy and gradient: the
    surviving quartets of a lattice cluster grow about as n^2.5 at 1..12
    waters."""
    return float(n_waters) ** 2.5


def sweep_shard(sizes: Sequence[int], rank: int, world: int) -> List[int]:
    """Molecules (indices into ``sizes``, waters per cluster) that ``rank``
    evaluates in a sweep sharded over ``world`` GPUs: contiguous and
    balanced by :func:`sweep_cost`, every molecule on exactly one rank."""
    return shard_by_cost([sweep_cost(n) for n in sizes], rank, world)


def _reduce_device() -> torch.device:
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Largest value of x over the ranks (x itself without a process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    """Sum of x over the ranks (x itself without a process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
