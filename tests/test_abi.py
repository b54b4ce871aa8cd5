"""C-ABI checks that need no GPU: the library builds, loads, exports every
entry point declared in include/*.h, and its host-only planner works."""

import ctypes
import glob
import os
import re

import numpy as np
import pytest

from qtqp_b200 import _lib, batch, problems
from qtqp_b200 import build as qbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
  names = set()
  for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
    text = open(hdr).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names |= set(re.findall(r"\b(qtqp_\w+)\s*\(", text))
  return sorted(names)


@pytest.fixture(scope="module")
def lib():
  qbuild.build()
  return _lib.load()


def test_library_exports_every_declared_symbol(lib):
  declared = _declared()
  assert declared, "no entry points found in include/"
  for name in declared:
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"
  assert set(_lib.EXPORTS) <= set(declared)


def test_version_and_last_error(lib):
  assert lib.qtqp_version() >= 1
  assert isinstance(lib.qtqp_last_error(), bytes)


def test_large_grid_is_one_block_per_b200_sm(lib):
  assert lib.qtqp_dense_large_blocks() == 148
  assert lib.qtqp_dense_large_workspace_bytes(4096, 8192) > 8 * 4096 * 8192
  assert lib.qtqp_dense_large_workspace_bytes(0, 8) == 0


def test_plan_orders_by_cost_and_sizes_workspace(lib):
  probs = [batch.DenseProblem(*_dense(problems.small_dense_instance(i))) for i in range(50)]
  hb = batch.HostBatch(probs, batch.SolveOptions())
  ns = hb.inst["n"][hb.order[:hb.count]]
  costs = hb.inst["m"][hb.order] * ns.astype(float) ** 2 + ns.astype(float) ** 3 / 3
  assert np.all(np.diff(costs) <= 0)
  assert sorted(hb.order.tolist()) == list(range(50))
  groups = hb.groups
  assert 1 <= len(groups) <= _lib.MAX_GROUPS
  assert sum(g[1] for g in groups) == 50 and groups[0][0] == 0
  for (b0, c0, _, _), (b1, _, _, _) in zip(groups, groups[1:]):
    assert b0 + c0 == b1  # groups tile the processing order
  for _, _, nt, smem in groups:
    assert nt in (32, 64, 128, 256) and 0 < smem <= 227 * 1024
  assert hb.workspace_bytes >= 256


def test_plan_large_instance_spills_to_global(lib):
  a = np.ones((400, 300))
  hb = batch.HostBatch([batch.DenseProblem(a, np.ones(400), np.ones(300), 10)],
                       batch.SolveOptions())
  assert hb.workspace_bytes > 8 * 400 * 300  # A (and the rest) in the global workspace


def test_plan_rejects_bad_instances(lib):
  inst = np.zeros(1, dtype=_lib.INSTANCE_DTYPE)
  inst["n"], inst["m"], inst["z"] = 3, 2, 2  # z == m: no inequality
  order = np.zeros(1, dtype=np.int32)
  plan = _lib.BatchPlan()
  opts = batch.SolveOptions().to_c()
  rc = lib.qtqp_dense_batch_plan(inst.ctypes.data, 1, ctypes.byref(opts), order.ctypes.data,
                                 0, 0, ctypes.byref(plan))
  assert rc == _lib.QTQP_ERR_BAD_ARG
  assert b"0 <= z < m" in lib.qtqp_last_error()
  rc = lib.qtqp_dense_batch_plan(inst.ctypes.data, 1, ctypes.byref(opts), order.ctypes.data,
                                 96, 0, ctypes.byref(plan))
  assert rc == _lib.QTQP_ERR_BAD_ARG


def test_kkt_workspace_size(lib):
  assert lib.qtqp_kkt_dense_workspace_bytes(0, 3) == 0
  assert lib.qtqp_kkt_dense_workspace_bytes(10, 20) > 8 * (10 * 20 + 10 * 10)


def _dense(prob):
  a, b, c, z, p = prob
  return a.toarray(), b, c, z, p.toarray()


def _band_inst(n, bw, m=None):
  inst = np.zeros(1, dtype=_lib.BAND_DTYPE)
  inst["n"], inst["m"], inst["z"], inst["bw"] = n, m or 2 * n, n // 4, bw
  inst["nnz_a"] = 4 * n
  return inst


def test_band_grid_partition_limits(lib):
  """Partition counts keep every interior at least bw long and stay within
  the grid; too-wide bands are refused."""
  inst = _band_inst(30000, 99)
  dp = lib.qtqp_band_grid_default_parts(inst.ctypes.data)
  assert 1 <= dp <= min(128, (30000 + 99) // 198)
  assert lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, dp) > 8 * 30000 * 100
  assert lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, 1) > 0
  assert lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, 128) > 0
  assert lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, 129) == 0
  assert lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, 0) == 0
  small = _band_inst(1000, 99)
  assert lib.qtqp_band_grid_workspace_bytes(small.ctypes.data, (1000 + 99) // 198) > 0
  assert lib.qtqp_band_grid_workspace_bytes(small.ctypes.data, (1000 + 99) // 198 + 1) == 0
  assert b"parts must be" in lib.qtqp_last_error()
  wide = _band_inst(30000, 127)
  assert lib.qtqp_band_grid_workspace_bytes(wide.ctypes.data, 4) == 0
  assert b"too wide" in lib.qtqp_last_error()


def test_band_grid_solve_rejects_bad_arguments(lib):
  """Argument errors of the whole-GPU banded entry point come back as
  QTQP_ERR_BAD_ARG with a message, before any device work."""
  inst = _band_inst(3000, 99)
  opts = batch.SolveOptions().to_c()
  ws_bytes = lib.qtqp_band_grid_workspace_bytes(inst.ctypes.data, 8)
  fake = 1 << 20  # a non-null device-looking address, never dereferenced
  def call(parts=8, pools=fake, ws=fake, nbytes=ws_bytes, o=ctypes.byref(opts)):
    return lib.qtqp_band_grid_solve(inst.ctypes.data, parts, pools, pools, pools, pools, pools,
                                    pools, pools, pools, None, ws, nbytes, o, None)
  assert call(parts=0) == _lib.QTQP_ERR_BAD_ARG
  assert b"parts must be" in lib.qtqp_last_error()
  assert call(pools=None) == _lib.QTQP_ERR_BAD_ARG
  assert b"null argument" in lib.qtqp_last_error()
  assert call(nbytes=ws_bytes - 1) == _lib.QTQP_ERR_BAD_ARG
  assert b"workspace smaller" in lib.qtqp_last_error()
  assert call(ws=fake + 8) == _lib.QTQP_ERR_BAD_ARG
  assert b"256-byte aligned" in lib.qtqp_last_error()
  bad = batch.SolveOptions().to_c()
  bad.max_iter = 0
  assert call(o=ctypes.byref(bad)) == _lib.QTQP_ERR_BAD_ARG
  assert b"invalid options" in lib.qtqp_last_error()


def test_sparse_grid_solve_rejects_bad_arguments(lib):
  """The supernodal whole-GPU entry point checks its plan against the
  instance and its pointers, sizes and options before any device work."""
  from qtqp_b200 import band, sparse
  a, b, c, z, p = problems.sparse_feasible(300, 320, 30, 4, per_row=2)
  plan = sparse.SparsePlan(a, p)
  prob = plan.permuted(a, b, c, z, p)
  pools = band.BandPools([prob], batch.SolveOptions())
  inst = np.ascontiguousarray(pools.inst[:1])
  desc = plan.desc
  ws_bytes = lib.qtqp_sparse_grid_workspace_bytes(inst.ctypes.data, ctypes.byref(desc))
  assert ws_bytes > 8 * desc.nvals
  assert lib.qtqp_sparse_grid_blocks() == desc.blocks
  opts = batch.SolveOptions().to_c()
  fake = 1 << 20  # a non-null device-looking address, never dereferenced
  def call(d=desc, pools_=fake, ws=fake, nbytes=ws_bytes, o=ctypes.byref(opts)):
    return lib.qtqp_sparse_grid_solve(inst.ctypes.data, ctypes.byref(d), pools_, pools_,
                                      pools_, pools_, pools_, pools_, pools_, pools_, pools_,
                                      pools_, None, ws, nbytes, o, None)
  assert call(pools_=None) == _lib.QTQP_ERR_BAD_ARG
  assert b"null argument" in lib.qtqp_last_error()
  assert call(nbytes=ws_bytes - 1) == _lib.QTQP_ERR_BAD_ARG
  assert b"workspace smaller" in lib.qtqp_last_error()
  assert call(ws=fake + 8) == _lib.QTQP_ERR_BAD_ARG
  assert b"16-byte aligned" in lib.qtqp_last_error()
  other = sparse.SparsePlan(*problems.sparse_feasible(301, 320, 30, 4, per_row=2)[::4]).desc
  assert call(d=other) == _lib.QTQP_ERR_BAD_ARG
  assert b"does not match" in lib.qtqp_last_error()
  warm = batch.SolveOptions(warm_corrections=2).to_c()
  assert call(o=ctypes.byref(warm)) == _lib.QTQP_ERR_BAD_ARG
  assert b"warm starts" in lib.qtqp_last_error()
  bad = batch.SolveOptions().to_c()
  bad.max_iter = 0
  assert call(o=ctypes.byref(bad)) == _lib.QTQP_ERR_BAD_ARG
  assert b"invalid options" in lib.qtqp_last_error()
