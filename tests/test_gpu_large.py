"""Parity of the large dense path (one QP on the whole GPU: grid-mode device
IPM, tensor-core Gram for the mixed factor) with the oracle and with the
per-block dense path, through the public API.

Criteria: identical SolutionStatus, the reference's acceptance conditions
(tests/kkt_checks.py), objective relative error <= 1e-6; the FP64 path also
takes the oracle's iteration count (+-1).
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


def _large_dense_like(n, m, z, rank, seed=1002):
  a, b, c, z, p = problems.large_dense(seed=seed, n=n, m=m, z=z, rank=rank)
  return a, b, c, z, p


def _solve(a, b, c, z, p, precision, **kw):
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p) if p is not None else None)
  return qb.solve_batch([q], storage="large", precision=precision, collect_stats=True, **kw)[0]


@pytest.mark.parametrize("shape", [(512, 1024, 128, 32), (300, 650, 40, 20), (129, 300, 1, 8)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_matches_oracle(shape, precision):
  n, m, z, rank = shape
  a, b, c, z, p = _large_dense_like(n, m, z, rank)
  sol = _solve(a, b, c, z, p, precision)
  ref = orc.solve(sp.csc_matrix(a), b, c, z, sp.csc_matrix(p), backend="dense")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
  if precision == "fp64":
    assert abs(len(sol.stats) - len(ref.stats)) <= 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_certificates(precision):
  a, b, c, z, p = problems.infeasible(300, 160, 30, seed=11)
  sol = _solve(a.toarray(), b, c, z, p.toarray(), precision)
  assert sol.status == qb.SolutionStatus.INFEASIBLE
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  a, b, c, z, p = problems.unbounded(300, 160, 30, seed=12)
  sol = _solve(a.toarray(), b, c, z, p.toarray(), precision)
  assert sol.status == qb.SolutionStatus.UNBOUNDED
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)


def test_large_and_block_paths_agree():
  a, b, c, z, p = _large_dense_like(200, 400, 50, 16, seed=7)
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p))
  s_large = qb.solve_batch([q], storage="large")[0]
  s_dense = qb.solve_batch([q], storage="dense")[0]
  assert s_large.status == s_dense.status == qb.SolutionStatus.SOLVED
  assert kkt_checks.objective_rel_err(s_large.x, s_dense.x, c, p) <= OBJ_TOL


def test_large_lp_without_p():
  a, b, c, z, p = problems.feasible(700, 300, 60, seed=5, density=0.3, lp=True)
  q = qb.QTQP(a=a, b=b, c=c, z=z)
  sol = qb.solve_batch([q], storage="large", precision="mixed")[0]
  ref = orc.solve(a, b, c, z, None, backend="dense")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, sp.csc_matrix((300, 300)), z)


def test_single_qp_solve_routes_to_the_large_path():
  a, b, c, z, p = _large_dense_like(320, 640, 64, 16, seed=3)
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p))
  assert q.storage_format(single=True) == "large"
  sol = q.solve(verbose=False)
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
