"""Sharding a batch of independent QPs over the GPUs of one node.

One process per GPU (``torch.distributed``; NCCL between GPUs, gloo for CPU
tests).  Instances are independent, so each rank solves its own share with
the single-GPU batch solver and the solutions are exchanged once at the end;
there is no collective on the data path.  Shares are balanced by an estimate
of each instance's work (the batch planner's cost m n^2 + n^3 / 3 of the
Gram product and Cholesky), since the sizes of a batch are uneven: n^3 ranges
over a factor of 500 in the batched workload.
"""

from __future__ import annotations

import heapq
from typing import Callable, List, Sequence


def instance_cost(n: int, m: int) -> float:
  """Work estimate of one QP: Gram product plus Cholesky flops."""
  return float(m) * n * n + float(n) ** 3 / 3.0


def shard_range(count: int, world: int, rank: int) -> range:
  """The contiguous, balanced slice of [0, count) owned by `rank` (the first
  count % world ranks take one extra instance)."""
  if world < 1 or not 0 <= rank < world:
    raise ValueError(f"rank {rank} outside a world of {world}")
  base, extra = divmod(count, world)
  start = rank * base + min(rank, extra)
  return range(start, start + base + (1 if rank < extra else 0))


def shard_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
  """Index lists (ascending) of a partition of range(len(costs)) into `world`
  shares of nearly equal total cost: largest first, each to the currently
  lightest share (ties to the lowest rank).  Deterministic, so every rank
  computes the same partition."""
  if world < 1:
    raise ValueError("world must be >= 1")
  order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
  heap = [(0.0, r) for r in range(world)]
  parts: List[List[int]] = [[] for _ in range(world)]
  for i in order:
    load, r = heapq.heappop(heap)
    parts[r].append(i)
    heapq.heappush(heap, (load + costs[i], r))
  return [sorted(p) for p in parts]


def solve_sharded(problems: Sequence, solve_fn: Callable | None = None, group=None,
                  balance: str = "cost", **solve_kwargs) -> List:
  """Solves `problems` across the ranks of `group` (default: the world) and
  returns every solution, in order, on every rank.

  balance: 'cost' (shares of equal estimated work; problems need n and m
  attributes) or 'count' (contiguous slices of equal length).
  solve_fn(list_of_problems, **solve_kwargs) -> list of solutions; default
  ``qtqp_b200.solve_batch`` on this rank's current GPU."""
  import torch.distributed as dist  # pylint: disable=g-import-not-at-top
  if solve_fn is None:
    from . import solve_batch as solve_fn  # pylint: disable=g-import-not-at-top
  world = dist.get_world_size(group)
  rank = dist.get_rank(group)
  if balance == "cost":
    parts = shard_by_cost([instance_cost(q.n, q.m) for q in problems], world)
  elif balance == "count":
    parts = [list(shard_range(len(problems), world, r)) for r in range(world)]
  else:
    raise ValueError(f"balance must be 'cost' or 'count', got {balance!r}")
  mine = parts[rank]
  local = list(solve_fn([problems[i] for i in mine], **solve_kwargs)) if mine else []
  if len(local) != len(mine):
    raise RuntimeError("solve_sharded: the solver returned a different number of solutions")
  gathered: list = [None] * world
  dist.all_gather_object(gathered, (mine, local), group=group)
  out: list = [None] * len(problems)
  for idx, sols in gathered:
    for i, s in zip(idx, sols):
      out[i] = s
  if any(s is None for s in out):
    raise RuntimeError("solve_sharded: a rank returned fewer solutions than its share")
  return out
