"""The allocation-free batch entry point (qtqp_dense_batch_solve_noalloc).

It serves callers that may not allocate device memory while solving (for
example code running inside another framework's memory pool, or a control
loop that must not touch the allocator once started): its scratch is a fixed
array inside the library instead of a caller-provided workspace.  These tests
call it through the C-ABI twice in a row and require the same results as the
workspace entry point, and check that a plan larger than the fixed array is
refused before anything is launched.

The file name sorts last, so pytest collects it after every other test file:
a run that stops at the first failure (-x) has then already run all the other
tests when one of these fails.  The tests also pass on their own in a fresh
process (the entry point looks the array's address up on its first call).
"""

import numpy as np
import pytest

from qtqp_b200 import _lib, batch, problems

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernel and arithmetic: results agree to rounding


def _dense(prob):
  a, b, c, z, p = prob
  return batch.DenseProblem(a.toarray(), b, c, z, p.toarray())


def _mixed_batch():
  """Small on-chip QPs plus two QPs whose A and P live in the scratch."""
  probs = [_dense(problems.small_dense_instance(i)) for i in range(24)]
  probs += [_dense(problems.feasible(220, 130, 12, s)) for s in (5, 6)]
  return batch.HostBatch(probs, batch.SolveOptions())


def _compare(got, ref):
  res, x, y, s, _ = got
  res_r, x_r, y_r, s_r, _ = ref
  np.testing.assert_array_equal(res["status"], res_r["status"])
  np.testing.assert_array_equal(res["iterations"], res_r["iterations"])
  for v, w in ((x, x_r), (y, y_r), (s, s_r)):
    np.testing.assert_allclose(v, w, rtol=TOL, atol=TOL, equal_nan=True)


def test_noalloc_matches_workspace_entry_point_on_two_calls():
  lib = _lib.load()
  hb = _mixed_batch()
  assert 256 < hb.workspace_bytes <= lib.qtqp_dense_batch_noalloc_max_workspace()
  ref = batch.DeviceBatch(hb)
  ref.upload()
  ref.launch()
  expected = ref.fetch()
  assert np.all(expected[0]["status"] == 0)
  db = batch.DeviceBatch(hb)
  db.upload()
  for _ in range(2):
    for t in (db.x, db.y, db.s):
      t.fill_(float("nan"))
    db.results.zero_()
    db.launch_noalloc()
    _compare(db.fetch(), expected)


def test_noalloc_refuses_plans_larger_than_its_scratch():
  lib = _lib.load()
  big = [_dense(problems.feasible(800, 700, 20, s, density=0.02)) for s in (1, 2)]
  hb = batch.HostBatch(big, batch.SolveOptions())
  assert hb.workspace_bytes > lib.qtqp_dense_batch_noalloc_max_workspace()
  db = batch.DeviceBatch(hb)
  db.upload()
  with pytest.raises(_lib.QtqpCudaError) as err:
    db.launch_noalloc()
  assert err.value.code == _lib.QTQP_ERR_BAD_ARG
  assert "16 MiB" in str(err.value)
