"""Sharding over ranks (world size 2, gloo on CPU): every instance is solved
exactly once, by the rank that owns it, and every rank gets all solutions in
order.  The shares are balanced by estimated work.  The solvers are
stand-ins that record which rank solved what, and one that runs the real
batch packing (HostBatch: pools, plan) on each rank's share with the device
step left out."""

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
    sols = distributed.solve_sharded(list(range(count)), solve_fn=fake_solve, scale=10,
                                     balance="count")
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


def test_shard_by_cost_partitions_and_balances():
  costs = [float(n) ** 3 for n in range(8, 65)] * 3
  for world in (1, 2, 3, 8):
    parts = distributed.shard_by_cost(costs, world)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    # largest-first greedy: within one largest item of the mean
    assert max(loads) - min(loads) <= max(costs)
  # contiguous equal-count slices of a cost-sorted list are far from balanced
  srt = sorted(costs, reverse=True)
  halves = [sum(srt[r] for r in distributed.shard_range(len(srt), 2, k)) for k in range(2)]
  bal = [sum(srt[i] for i in p) for p in distributed.shard_by_cost(srt, 2)]
  assert max(bal) / min(bal) < max(halves) / min(halves)


def _packing_worker(rank, world, port, count, out_q):
  os.environ["MASTER_ADDR"] = "127.0.0.1"
  os.environ["MASTER_PORT"] = str(port)
  dist.init_process_group("gloo", rank=rank, world_size=world)
  try:
    import numpy as np
    import qtqp_b200 as qb
    from qtqp_b200 import batch, problems

    def pack_only(qps):
      """solve_batch's host side on this rank's share: HostBatch packs the
      pools and plans; the device step is left out.  Returns, per problem,
      its A read back from the packed pool."""
      hb = batch.HostBatch(qps, batch.SolveOptions())
      out = []
      for j, q in enumerate(qps):
        d = hb.inst[j]
        a0, m, n = int(d["a_off"]), int(d["m"]), int(d["n"])
        out.append((rank, hb.a_pool[a0:a0 + m * n].reshape(n, m).T.copy()))
      assert hb.plan.num_groups >= 1 and hb.workspace_bytes >= 256
      return out

    qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in
           (problems.small_dense_instance(i) for i in range(count))]
    res = distributed.solve_sharded(qps, solve_fn=pack_only)
    for q, (_, a) in zip(qps, res):
      np.testing.assert_array_equal(a, q.a.toarray())
    owners = [o for o, _ in res]
    costs = [distributed.instance_cost(q.n, q.m) for q in qps]
    load = [sum(c for c, o in zip(costs, owners) if o == r) for r in range(world)]
    out_q.put((rank, owners, load))
  finally:
    dist.destroy_process_group()


def test_solve_sharded_packs_each_share_on_its_rank():
  world, count = 2, 40
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_packing_worker, args=(r, world, port, count, q))
           for r in range(world)]
  for p in procs:
    p.start()
  results = [q.get(timeout=180) for _ in range(world)]
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  owners0 = results[0][1]
  assert all(r[1] == owners0 for r in results)  # every rank agrees on the owners
  assert set(owners0) == {0, 1}
  load = results[0][2]
  assert max(load) / min(load) < 1.2
