"""Sparse QPs whose Gram matrix is narrow-banded only after reordering: the
variables of stage-ordered MPC QPs are shuffled, the library finds a reverse
Cuthill-McKee ordering, solves the reordered QP on the banded device paths
(a batch, and one QP on the whole GPU) and maps x back.  Checked against the
oracle (SuperLU, the reference's SCIPY backend algorithm) on the shuffled QP:
the same status and iteration count within one, objective within 1e-6, the
reference's acceptance conditions.
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


def _shuffled_mpc(horizon, seed, nx=40, nu=20):
  a, b, c, z, p = problems.mpc_feasible(horizon, seed=1003 + seed, nx=nx, nu=nu)
  perm = np.random.default_rng(seed).permutation(a.shape[1])
  return qb.QTQP(a=sp.csc_matrix(a[:, perm]), b=b, c=c[perm], z=z,
                 p=sp.csc_matrix(p[perm][:, perm]))


def _check(q, sol):
  ref = orc.solve(q.a, q.b, q.c, q.z, q.p, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, q.a, q.b, q.c, q.p, q.z)
  assert abs(len(sol.stats) - len(ref.stats)) <= 1
  f = q.c @ sol.x + 0.5 * sol.x @ (q.p @ sol.x)
  fr = q.c @ ref.x + 0.5 * ref.x @ (q.p @ ref.x)
  assert abs(f - fr) <= OBJ_TOL * max(1.0, abs(fr))


def test_reordered_batch_matches_oracle():
  qps = [_shuffled_mpc(12, s) for s in range(4)]  # n = 720: the reordered band fits n / 4
  assert all(q.storage_format() == "band" and q.band_permutation() is not None for q in qps)
  sols = qb.solve_batch(qps, collect_stats=True)
  for q, s in zip(qps, sols):
    _check(q, s)


def test_reordered_single_qp_on_the_whole_gpu_matches_oracle():
  q = _shuffled_mpc(40, 7, nx=20, nu=10)  # n = 1200; reordered half-bandwidth within 118
  assert q.storage_format(single=True) == "band_grid"
  _check(q, q.solve(verbose=False, collect_stats=True))
