"""Benchmark configurations at their stated sizes against the reference's own
results (tests/golden/reference_configs.npz, recorded from the reference with
SCIPY_DENSE for the large dense QP and SCIPY for the parametric family):

* the large dense QP (n=4096, m=8192, z=1024) on the whole-GPU path, in FP64
  and in mixed precision: the reference's status, objective within 1e-6
  relative, the reference's acceptance conditions, and (FP64) the
  reference's iteration count within one;
* 32 held-out instances (16384..16415) of the T=50 parametric MPC family
  (n=3000, m=8000): the reference's statuses and objectives through the plain
  batched path and through the learned warm start (a network trained on the
  plain method's solutions of instances 0..1023; rejected predictions start
  the plain method cold, or from the prediction with warm_shift), whose
  statuses must also equal the plain path's.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import qtqp_b200 as qb
from qtqp_b200 import problems, warmstart
from tests import golden_io, kkt_checks

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6  # relative objective error against the reference
WARM_CORRECTIONS = 8


def _golden():
  return golden_io.load("reference_configs.npz")


def _objective(q, x):
  return float(q.c @ x + 0.5 * x @ (q.p @ x))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_dense_full_size_matches_reference(precision):
  g = _golden()
  a, b, c, z, p = problems.large_dense()
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p))
  assert q.storage_format(single=True) == "large"
  sol = q.solve(precision=precision, verbose=False, collect_stats=True)
  assert sol.status.value == str(g["large_dense/status"])
  ref = float(g["large_dense/objective"])
  assert abs(_objective(q, sol.x) - ref) <= OBJ_TOL * max(1.0, abs(ref))
  kkt_checks.assert_status_certificate(sol, q.a, q.b, q.c, q.p, z)
  if precision == "fp64":
    assert abs(len(sol.stats) - int(g["large_dense/iters"])) <= 1


def _family():
  fam = problems.parametric_mpc_family()
  def qp(i):
    a, b, c, z, p = problems.parametric_mpc_instance(fam, i)
    return qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  return fam[-1], qp


def test_parametric_t50_plain_and_warm_started_match_reference():
  g = _golden()
  idx = [int(i) for i in g["parametric/index"]]
  ref_status = [str(s) for s in g["parametric/status"]]
  ref_obj = g["parametric/objective"]
  thetas, qp = _family()
  test_qps = [qp(i) for i in idx]
  assert all(q.storage_format() == "band" for q in test_qps)
  plain = qb.solve_batch(test_qps)
  for q, s, st, fo in zip(test_qps, plain, ref_status, ref_obj):
    assert s.status.value == st
    kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)
    if st == "solved":
      assert abs(_objective(q, s.x) - fo) <= OBJ_TOL * max(1.0, abs(fo))
  # Learned warm start: train on the plain method's solutions of 0..1023.
  train_qps = [qp(i) for i in range(1024)]
  sols = qb.solve_batch(train_qps)
  keep = [i for i, s in enumerate(sols) if s.status == qb.SolutionStatus.SOLVED]
  assert len(keep) > 0.95 * len(train_qps)
  q0 = test_qps[0]
  targets = warmstart.targets_from(q0.n, q0.z, [sols[i].x for i in keep],
                                   [sols[i].y for i in keep], [sols[i].s for i in keep])
  net = warmstart.WarmStartMLP(dim=thetas.shape[1], n=q0.n, m=q0.m, z=q0.z, seed=0)
  net.train(thetas[keep], targets, epochs=30, batch=64, lr=2e-3)
  net.calibrate(thetas[keep], targets)
  for shift in (0.0, 0.1):  # 0.1: a rejected prediction starts the IPM at the prediction
    warm = qb.solve_batch(test_qps, warm_start=(net, thetas[idx]),
                          warm_corrections=WARM_CORRECTIONS, warm_shift=shift)
    for q, s, sp_, st, fo in zip(test_qps, warm, plain, ref_status, ref_obj):
      assert s.status == sp_.status
      assert s.status.value == st
      kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)
      if st == "solved":
        assert abs(_objective(q, s.x) - fo) <= OBJ_TOL * max(1.0, abs(fo))
