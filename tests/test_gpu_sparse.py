"""Parity of the supernodal path (one sparse QP on the whole GPU: grid-mode
device IPM with a supernodal Cholesky of the Gram matrix) with the oracle's
sparse-LU backend (the reference's SCIPY backend restated), through the
public API.

Criteria, as for the other paths: identical SolutionStatus, the reference's
acceptance conditions (tests/kkt_checks.py), objective relative error <= 1e-6;
the FP64 form also takes the oracle's iteration count (+-1).  Families: random
sparse rows (two or three entries per row) with and without P, a min-cost
flow on a grid network, and sparse infeasible / unbounded certificates.
"""

import numpy as np
import pytest

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import problems
from tests import kkt_checks

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6


def _solve(a, b, c, z, p, precision="fp64", **kw):
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  return q, qb.solve_batch([q], storage="sparse", precision=precision, collect_stats=True,
                           **kw)[0]


@pytest.mark.parametrize("shape", [(600, 700, 60, 2), (1000, 1000, 100, 2), (400, 600, 40, 3)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sparse_matches_oracle(shape, precision):
  n, m, z, per_row = shape
  a, b, c, z, p = problems.sparse_feasible(n, m, z, 31 + n, per_row=per_row)
  _, sol = _solve(a, b, c, z, p, precision)
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
  if precision == "fp64":
    assert abs(len(sol.stats) - len(ref.stats)) <= 1


def test_sparse_lp_and_no_equilibration():
  a, b, c, z, p = problems.sparse_feasible(500, 600, 50, 7, per_row=2, lp=True)
  q = qb.QTQP(a=a, b=b, c=c, z=z)
  sol = qb.solve_batch([q], storage="sparse")[0]
  ref = orc.solve(a, b, c, z, None, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  a, b, c, z, p = problems.sparse_feasible(500, 600, 50, 8, per_row=2)
  q, sol = _solve(a, b, c, z, p, equilibrate=False)
  ref = orc.solve(a, b, c, z, p, backend="superlu", equilibrate=False)
  assert sol.status.value == ref.status
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL


def test_grid_flow_sparse_and_band_paths_agree():
  a, b, c, z, p = problems.grid_flow(16)
  q, s_sparse = _solve(a, b, c, z, p)
  s_band = qb.solve_batch([q], storage="band")[0]
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert s_sparse.status.value == s_band.status.value == ref.status == "solved"
  kkt_checks.assert_status_certificate(s_sparse, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(s_sparse.x, ref.x, c, p) <= OBJ_TOL
  assert kkt_checks.objective_rel_err(s_sparse.x, s_band.x, c, p) <= OBJ_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sparse_certificates(precision):
  a, b, c, z, p = problems.sparse_infeasible(500, 700, 50, 21)
  _, sol = _solve(a, b, c, z, p, precision)
  assert sol.status == qb.SolutionStatus.INFEASIBLE
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  a, b, c, z, p = problems.sparse_unbounded(500, 700, 50, 22)
  _, sol = _solve(a, b, c, z, p, precision)
  assert sol.status == qb.SolutionStatus.UNBOUNDED
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)


def test_auto_routing_and_reproducibility():
  """A grid-network QP whose band is too wide for the partitioned band path
  goes to the supernodal path when solved on its own; two solves give
  identical bits (no atomics in the factor)."""
  a, b, c, z, p = problems.grid_flow(32)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format(single=True) == "sparse"
  s1 = q.solve(verbose=False)
  s2 = q.solve(verbose=False)
  assert s1.status == qb.SolutionStatus.SOLVED
  assert np.array_equal(s1.x, s2.x) and np.array_equal(s1.y, s2.y)
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert kkt_checks.objective_rel_err(s1.x, ref.x, c, p) <= OBJ_TOL


@pytest.mark.parametrize("case", ["grid_flow_40", "random_3000"])
def test_larger_sparse_qps_match_oracle(case):
  """Sizes whose top levels split their row slabs' update lists and their
  forward gathers over several blocks (long update lists, few slabs)."""
  if case == "grid_flow_40":
    a, b, c, z, p = problems.grid_flow(40)
  else:
    a, b, c, z, p = problems.sparse_feasible(3000, 3000, 300, 77, per_row=2)
  q, sol = _solve(a, b, c, z, p)
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
  assert abs(len(sol.stats) - len(ref.stats)) <= 1
