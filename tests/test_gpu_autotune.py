"""The launch-shape autotuner (qtqp_b200.autotune; no reference counterpart).

Tuning a batch's launch groups returns valid table entries, and a solve
planned with the tuned table gives the same statuses as the default plan,
with results that pass the reference's acceptance conditions and agree in
objective to 1e-6 (different launch shapes only change reduction orders).
"""

import json

import numpy as np
import pytest

import qtqp_b200 as qb
from qtqp_b200 import autotune, batch, problems
from tests import kkt_checks

pytestmark = pytest.mark.gpu


def _qps(count):
  return [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in
          (problems.small_dense_instance(i) for i in range(count))]


def test_tuned_plan_matches_default_plan(tmp_path):
  qps = _qps(600)
  table = autotune.tune_dense_batch(qps, reps=1)
  for e in table:
    assert e["block_threads"] in (32, 64, 128, 256) and e["lean"] in (0, 1)
    assert e["onchip"] in (0, 1) and e["n_lo"] <= e["n_hi"]
    # The whole batch (groups running concurrently) is not slower with the
    # table than with the default plan, within the spread of repeated
    # timings; a group alone may be.
    assert e["batch_ms"] <= 1.05 * e["batch_default_ms"]
  default = qb.solve_batch(qps, tuning=None)
  tuned = qb.solve_batch(qps, tuning=table)
  for q, sd, st in zip(qps, default, tuned):
    assert sd.status == st.status
    kkt_checks.assert_status_certificate(st, q.a, q.b, q.c, q.p, q.z)
    fd = q.c @ sd.x + 0.5 * sd.x @ (q.p @ sd.x)
    ft = q.c @ st.x + 0.5 * st.x @ (q.p @ st.x)
    assert abs(fd - ft) <= 1e-6 * max(1.0, abs(fd))
  path = str(tmp_path / "tuning.json")
  autotune.save(table, path=path)
  assert autotune.load(path=path) == json.loads(json.dumps(table))


def test_every_candidate_shape_solves_the_same():
  qps = _qps(64)
  hb = batch.HostBatch(qps, batch.SolveOptions(), pinned=True)
  db = batch.DeviceBatch(hb)
  db.upload()
  db.launch()
  ref = db.fetch()[0]["status"].copy()
  n_hi = int(hb.inst["n"].max())
  for nt, lean, onchip in autotune.CANDIDATES + autotune.SMALL_CANDIDATES:
    hb.replan([{"n_lo": 0, "n_hi": n_hi, "block_threads": nt, "lean": lean,
                "onchip": onchip}])
    db.refresh_plan()
    db.launch()
    got = db.fetch()[0]["status"]
    np.testing.assert_array_equal(got, ref)


def test_batch_pass_keeps_statuses():
  """The optional pass over the whole concurrent batch returns a table that
  solves every instance with the default plan's status."""
  qps = _qps(300)
  table = autotune.tune_dense_batch(qps, reps=1, batch_pass=True)
  for e in table:
    assert e["block_threads"] in (32, 64, 128, 256)
    assert e["batch_ms"] > 0.0 and e["batch_default_ms"] > 0.0
  default = qb.solve_batch(qps, tuning=None)
  tuned = qb.solve_batch(qps, tuning=table)
  assert [s.status for s in default] == [s.status for s in tuned]
