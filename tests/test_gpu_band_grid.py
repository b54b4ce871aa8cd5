"""Parity of the whole-GPU banded solve (one cooperative launch, partitioned
band factorisation over interiors and separators) with the oracle and with
the one-block banded path.

Criteria as for the other device paths: identical SolutionStatus, the
reference's acceptance conditions, objective relative error <= 1e-6.
"""

import pytest

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import band, batch, problems
from tests import kkt_checks

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6


def _grid_solve(q, precision="fp64", parts=None):
  """Device solve of q on the whole GPU with a given partition count."""
  hb = band.HostBandBatch([q.band_problem()], batch.SolveOptions(precision=precision))
  dg = band.DeviceBandGrid(hb, parts=parts)
  dg.upload()
  dg.launch()
  res, x, y, s, _ = dg.fetch()
  return res[0], x, y, s, dg.parts


def _assert_feasible(x, y, s, a, b, c, p):
  e = kkt_checks.kkt_errors(x, y, s, a, b, c, p)
  assert e["pres"] < 1e-7 + 1e-8 * e["prel"], e
  assert e["dres"] < 1e-7 + 1e-8 * e["drel"], e


@pytest.mark.parametrize("horizon", [20, 50])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_grid_matches_oracle_on_mpc(horizon, precision):
  a, b, c, z, p = problems.mpc_feasible(horizon)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format(single=True) == "band_grid"
  sol = qb.solve_batch([q], storage="band_grid", precision=precision, collect_stats=True)[0]
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
  if precision == "fp64":
    assert abs(len(sol.stats) - len(ref.stats)) <= 1


@pytest.mark.parametrize("parts", [1, 2, 3, 7, 15])
def test_grid_partition_counts_agree(parts):
  """Every partition count (1 = one interior, no separator; 15 = the most
  that keeps interiors >= bw at T=50) gives the one-block path's solution."""
  a, b, c, z, p = problems.mpc_feasible(50)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  ref = qb.solve_batch([q], storage="band")[0]
  res, x, y, s, used = _grid_solve(q, parts=parts)
  assert used == parts
  assert int(res["status"]) == 0 and int(res["error"]) == 0
  _assert_feasible(x, y, s, a, b, c, p)
  assert kkt_checks.objective_rel_err(x, ref.x, c, p) <= OBJ_TOL


@pytest.mark.parametrize("parts", [4, 33, 99])
def test_grid_narrow_band_ragged_partitions(parts):
  """nx=4, nu=2 (half-bandwidth 9), n = 1794: interiors of uneven length,
  up to 98 separators in the chain."""
  a, b, c, z, p = problems.mpc_feasible(299, nx=4, nu=2, seed=7)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert band.gram_bandwidth(q.a, q.p) == 9
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert ref.status == "solved"
  for precision in ("fp64", "mixed"):
    res, x, y, s, _ = _grid_solve(q, precision=precision, parts=parts)
    assert int(res["status"]) == 0
    _assert_feasible(x, y, s, a, b, c, p)
    assert kkt_checks.objective_rel_err(x, ref.x, c, p) <= OBJ_TOL


def test_grid_infeasible_mpc():
  """Contradictory bounds (x_0 fixed outside its box) give a certificate."""
  a, b, c, z, p = problems.mpc_feasible(30)
  b = b.copy()
  b[0] = 50.0
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  sol = qb.solve_batch([q], storage="band_grid")[0]
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status == "infeasible"
  kkt_checks.assert_infeasible(sol, a, b, z)


def test_grid_full_size_mpc():
  """The T=500 MPC QP (n=30000, m=80000) through QTQP.solve."""
  a, b, c, z, p = problems.mpc_t500()
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format(single=True) == "band_grid"
  sol = q.solve(verbose=False)
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  assert sol.status.value == ref.status == "solved"
  kkt_checks.assert_solved(sol, a, b, c, p, z)
  assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL


def test_grid_tiny_band_short_interiors():
  """Half-bandwidth 2 with the default 128 partitions: interiors of about 7
  columns, shorter than one 8-column panel."""
  a, b, c, z, p = problems.mpc_feasible(600, nx=1, nu=1, seed=13)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert band.gram_bandwidth(q.a, q.p) == 2
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  res, x, y, s, parts = _grid_solve(q)
  assert parts == 128
  assert int(res["status"]) == 0 and ref.status == "solved"
  _assert_feasible(x, y, s, a, b, c, p)
  assert kkt_checks.objective_rel_err(x, ref.x, c, p) <= OBJ_TOL


def test_grid_wide_band():
  """nx=40, nu=36: half-bandwidth 115, near the widest band whose separator
  blocks fit in shared memory."""
  a, b, c, z, p = problems.mpc_feasible(20, nx=40, nu=36, seed=17)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert band.gram_bandwidth(q.a, q.p) == 115
  assert q.storage_format(single=True) == "band_grid"
  ref = orc.solve(a, b, c, z, p, backend="superlu")
  sol = qb.solve_batch([q], storage="band_grid")[0]
  assert sol.status.value == ref.status
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  if ref.status == "solved":
    assert kkt_checks.objective_rel_err(sol.x, ref.x, c, p) <= OBJ_TOL
