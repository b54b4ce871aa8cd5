"""Sharding a batch of independent QPs over the GPUs of one node.

One process per GPU (``torch.distributed``; NCCL between GPUs, gloo for CPU
tests).  Instances are independent, so each rank solves a contiguous slice
with the single-GPU batch solver and the solutions are exchanged once at the
end; there is no collective on the data path.
"""

from __future__ import annotations

from typing import Callable, List, Sequence


def shard_range(count: int, world: int, rank: int) -> range:
  """The contiguous, balanced slice of [0, count) owned by `rank` (the first
  count % world ranks take one extra instance)."""
  if world < 1 or not 0 <= rank < world:
    raise ValueError(f"rank {rank} outside a world of {world}")
  base, extra = divmod(count, world)
  start = rank * base + min(rank, extra)
  return range(start, start + base + (1 if rank < extra else 0))


def solve_sharded(problems: Sequence, solve_fn: Callable | None = None, group=None,
                  **solve_kwargs) -> List:
  """Solves `problems` across the ranks of `group` (default: the world) and
  returns every solution, in order, on every rank.

  solve_fn(list_of_problems, **solve_kwargs) -> list of solutions; default
  ``qtqp_b200.solve_batch`` on this rank's current GPU."""
  import torch.distributed as dist  # pylint: disable=g-import-not-at-top
  if solve_fn is None:
    from . import solve_batch as solve_fn  # pylint: disable=g-import-not-at-top
  world = dist.get_world_size(group)
  rank = dist.get_rank(group)
  mine = shard_range(len(problems), world, rank)
  local = list(solve_fn([problems[i] for i in mine], **solve_kwargs)) if len(mine) else []
  gathered: list = [None] * world
  dist.all_gather_object(gathered, (mine.start, local), group=group)
  out: list = [None] * len(problems)
  for start, sols in gathered:
    for k, s in enumerate(sols):
      out[start + k] = s
  if any(s is None for s in out):
    raise RuntimeError("solve_sharded: a rank returned fewer solutions than its shard")
  return out
