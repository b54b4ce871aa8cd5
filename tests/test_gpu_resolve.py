"""Re-solves (no reference counterpart beyond tests/test_qtqp.py:1578-1598,
where solve() is called twice on one problem and both results agree).

* The reference's own check: solve() twice on one QTQP gives the same status
  and objective.
* Re-solves started from earlier solutions (solve_batch(initial=...), the
  device IPM started from a given point): against the oracle's interior-point
  method started from the identical point (status, iteration count within
  one, objective within 1e-6), and on a nearby QP (perturbed b, c) the same
  status as its cold solve with fewer iterations.
"""

import numpy as np
import pytest

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import batch, problems
from tests import kkt_checks

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6
SHIFT = 0.1


def _objective(q, x):
  return float(q.c @ x + 0.5 * x @ (q.p @ x))


def test_solve_twice_on_one_problem_agrees():
  a, b, c, z, p = problems.feasible(30, 10, 5, 42)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  s1 = q.solve(verbose=False)
  s2 = q.solve(verbose=False)
  assert s1.status == s2.status == qb.SolutionStatus.SOLVED
  kkt_checks.assert_solved(s1, a, b, c, p, z)
  np.testing.assert_allclose(_objective(q, s1.x), _objective(q, s2.x), rtol=1e-5, atol=1e-5)


def _batch(count=24):
  return [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in
          (problems.small_dense_instance(i) for i in range(count))]


def test_resolve_from_solutions_matches_oracle_from_same_point():
  qps = _batch()
  cold = qb.solve_batch(qps, collect_stats=True)
  warm = qb.solve_batch(qps, initial=cold, initial_shift=SHIFT, collect_stats=True)
  hb = batch.HostBatch(qps, batch.SolveOptions())
  x0, y0, s0 = batch.start_points(hb, qps, cold, SHIFT)
  for j, (q, sc, sw) in enumerate(zip(qps, cold, warm)):
    d = hb.inst[j]
    n0, m0 = int(d["n_off"]), int(d["m_off"])
    init = (x0[n0:n0 + q.n], y0[m0:m0 + q.m], s0[m0:m0 + q.m])
    ref = orc.solve(q.a, q.b, q.c, q.z, q.p, backend="dense", init=init)
    assert sw.status.value == ref.status == sc.status.value
    kkt_checks.assert_status_certificate(sw, q.a, q.b, q.c, q.p, q.z)
    assert abs(len(sw.stats) - len(ref.stats)) <= 1
    fr = _objective(q, ref.x)
    assert abs(_objective(q, sw.x) - fr) <= OBJ_TOL * max(1.0, abs(fr))


def test_resolve_of_nearby_problems_needs_fewer_iterations():
  qps = _batch(64)
  cold = qb.solve_batch(qps, collect_stats=True)
  rng = np.random.default_rng(7)
  near = []
  for q in qps:
    b = q.b + 1e-3 * rng.normal(size=q.m) * (1 + np.abs(q.b))
    c = q.c + 1e-3 * rng.normal(size=q.n) * (1 + np.abs(q.c))
    near.append(qb.QTQP(a=q.a, b=b, c=c, z=q.z, p=q.p))
  near_cold = qb.solve_batch(near, collect_stats=True)
  near_warm = qb.solve_batch(near, initial=cold, collect_stats=True)
  for q, sc, sw in zip(near, near_cold, near_warm):
    assert sw.status == sc.status
    kkt_checks.assert_status_certificate(sw, q.a, q.b, q.c, q.p, q.z)
  it_cold = sum(len(s.stats) for s in near_cold)
  it_warm = sum(len(s.stats) for s in near_warm)
  assert it_warm < it_cold, (it_warm, it_cold)


def test_initial_points_are_checked():
  qps = _batch(3)
  with pytest.raises(ValueError):
    qb.solve_batch(qps, initial=[None, None])
  bad = (np.zeros(qps[0].n + 1), np.zeros(qps[0].m), np.zeros(qps[0].m))
  with pytest.raises(ValueError):
    qb.solve_batch(qps, initial=[bad, None, None])
