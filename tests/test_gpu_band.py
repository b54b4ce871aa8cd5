"""Parity of the banded/sparse device IPM (stage-ordered MPC problems) with
the oracle and with the dense device path, through the public API.

Criteria as for the dense path: identical SolutionStatus, the reference's
acceptance conditions, objective relative error <= 1e-6.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import problems
from tests import kkt_checks

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6


def _qp(horizon, seed=1003):
  a, b, c, z, p = problems.mpc_feasible(horizon, seed=seed)
  return qb.QTQP(a=a, b=b, c=c, z=z, p=p), (a, b, c, z, p)


@pytest.mark.parametrize("horizon", [3, 10, 25])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_band_matches_oracle_on_mpc(horizon, precision):
  q, (a, b, c, z, p) = _qp(horizon)
  assert q.storage_format() == ("band" if horizon >= 10 else "dense")
  sol = qb.solve_batch([q], storage="band", precision=precision, collect_stats=True)[0]
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
  if precision == "fp64":
    assert abs(len(sol.stats) - len(ref.stats)) <= 1


def test_band_and_dense_paths_agree():
  q, (a, b, c, z, p) = _qp(6)
  s_band = qb.solve_batch([q], storage="band")[0]
  s_dense = qb.solve_batch([q], storage="dense")[0]
  assert s_band.status == s_dense.status == qb.SolutionStatus.SOLVED
  assert kkt_checks.objective_rel_err(s_band.x, s_dense.x, c, p) <= OBJ_TOL


def test_band_batch_of_parametric_instances():
  """The parametric family: same A, P; (b, c) perturbed per instance."""
  fam = problems.parametric_mpc_family(count=24, horizon=8)
  qps, refs = [], []
  for i in range(24):
    a, b, c, z, p = problems.parametric_mpc_instance(fam, i)
    qps.append(qb.QTQP(a=a, b=b, c=c, z=z, p=p))
    refs.append(orc.solve(a, b, c, z, p, backend="superlu"))
  sols = qb.solve_batch(qps, storage="band")
  for q, s, r in zip(qps, sols, refs):
    assert s.status.value == r.status
    kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)
    if r.status == "solved":
      assert kkt_checks.objective_rel_err(s.x, r.x, q.c, q.p) <= OBJ_TOL


def test_band_infeasible_mpc():
  """Contradictory bounds (x_0 fixed outside its box) give a certificate."""
  a, b, c, z, p = problems.mpc_feasible(5)
  b = b.copy()
  b[0] = 50.0  # x_0[0] = 50 but |x_0[0]| <= 5
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  sol = qb.solve_batch([q], storage="band")[0]
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status == "infeasible"
  kkt_checks.assert_infeasible(sol, a, b, z)


def test_band_lp_without_p():
  a, b, c, z, p = problems.mpc_feasible(6)
  q = qb.QTQP(a=a, b=b, c=c, z=z)  # LP: box constraints bound it
  sol = qb.solve_batch([q], storage="band")[0]
  ref = orc.solve(a, b, c, z, None, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, sp.csc_matrix(p.shape), z)


@pytest.mark.parametrize("nx,nu,horizon", [(2, 1, 60), (4, 2, 40), (1, 1, 120)])
def test_band_narrow_bands(nx, nu, horizon):
  """Half-bandwidths 4, 9 and 2: bands narrower than the band kernels'
  8-column panels and solve blocks."""
  a, b, c, z, p = problems.mpc_feasible(horizon, nx=nx, nu=nu, seed=11)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format() == "band"
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  for precision in ("fp64", "mixed"):
    sol = qb.solve_batch([q], storage="band", precision=precision)[0]
    assert sol.status.value == ref.status
    kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
    if ref.status == "solved":
      assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
