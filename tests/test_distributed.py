"""Sharding over ranks (world size 2, gloo on CPU): every instance is solved
exactly once, by the rank that owns it, and every rank gets all solutions in
order.  The solver is a stand-in that records which rank solved what."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from qtqp_b200 import distributed


def _free_port():
  with socket.socket() as s:
    s.bind(("127.0.0.1", 0))
    return s.getsockname()[1]


@pytest.mark.parametrize("count,world", [(10, 2), (3, 2), (1, 2), (0, 2), (7, 3)])
def test_shard_ranges_partition(count, world):
  seen = []
  for r in range(world):
    rg = distributed.shard_range(count, world, r)
    seen.extend(rg)
    assert len(rg) in (count // world, count // world + 1)
  assert seen == list(range(count))


def test_shard_range_rejects_bad_rank():
  with pytest.raises(ValueError):
    distributed.shard_range(4, 2, 2)


def _worker(rank, world, port, count, out_q):
  os.environ["MASTER_ADDR"] = "127.0.0.1"
  os.environ["MASTER_PORT"] = str(port)
  dist.init_process_group("gloo", rank=rank, world_size=world)
  try:
    def fake_solve(probs, scale):
      return [(p * scale, rank) for p in probs]
    sols = distributed.solve_sharded(list(range(count)), solve_fn=fake_solve, scale=10)
    out_q.put((rank, sols))
  finally:
    dist.destroy_process_group()


@pytest.mark.parametrize("count", [9, 1])
def test_solve_sharded_two_ranks(count):
  world = 2
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, world, port, count, q)) for r in range(world)]
  for p in procs:
    p.start()
  results = dict(q.get(timeout=120) for _ in range(world))
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  for rank in range(world):
    sols = results[rank]
    assert [v for v, _ in sols] == [10 * i for i in range(count)]
    owners = [o for _, o in sols]
    for r in range(world):
      assert [i for i, o in enumerate(owners) if o == r] == list(
          distributed.shard_range(count, world, r))
