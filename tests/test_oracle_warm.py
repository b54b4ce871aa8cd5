"""The oracle's restatement of the warm-start attempt (CPU only).

A prediction equal to the plain method's own solution is accepted without a
correction; a prediction with rows flipped in the active set is rejected by
the termination test, and the correction rounds repair it; an infeasible QP
is never accepted; an accepted answer matches the plain solution.
"""

import numpy as np
import pytest

from oracle import qtqp_oracle as orc
from qtqp_b200 import problems


def _case(seed, m=60, n=30, z=6):
  a, b, c, z, p = problems.feasible(m, n, z, seed)
  plain = orc.solve(a, b, c, z, p, backend="superlu")
  assert plain.status == orc.STATUS_SOLVED
  act = plain.y > plain.s
  act[:z] = True
  return (a, b, c, z, p), plain, act


@pytest.mark.parametrize("seed", [3, 11, 29])
@pytest.mark.parametrize("backend", ["superlu", "dense"])
def test_true_active_set_is_accepted(seed, backend):
  qp, plain, act = _case(seed)
  r = orc.warm_try(*qp, plain.x, plain.y, act, backend=backend)
  assert r.accepted and r.rounds == 1
  a, b, c, z, p = qp
  obj = lambda x: c @ x + 0.5 * x @ (p @ x)
  assert abs(obj(r.x) - obj(plain.x)) <= 1e-6 * max(1.0, abs(obj(plain.x)))
  np.testing.assert_allclose(a @ r.x + r.s, b, atol=1e-6 * max(1.0, np.abs(b).max()))
  assert np.all(r.y[z:] >= 0.0) and np.all(r.s[z:] >= 0.0) and np.all(r.s[:z] == 0.0)


@pytest.mark.parametrize("seed", [5, 6, 7, 8])
def test_flipped_rows_are_repaired_by_corrections(seed):
  """One active row predicted free is rejected as it stands and repaired by
  the primal-dual corrections; so is one strictly inactive row predicted
  tight.  (P is low-rank here, so a wrong row moves the reduced solution
  far and the repair takes a few rounds.)"""
  qp, plain, act = _case(seed, m=30, n=60, z=5)
  z = qp[3]
  gap = np.abs(plain.y - plain.s)
  on = np.nonzero(act & (np.arange(act.size) >= z) & (gap > 1e-3))[0]
  off = np.nonzero(~act & (gap > 1e-3))[0]
  assert on.size and off.size
  dropped = act.copy()
  dropped[on[0]] = False
  r0 = orc.warm_try(*qp, plain.x, plain.y, dropped, corrections=0)
  assert not r0.accepted and r0.rounds == 1
  r = orc.warm_try(*qp, plain.x, plain.y, dropped, corrections=8)
  assert r.accepted and 2 <= r.rounds <= 9
  added = act.copy()
  added[off[0]] = True
  r = orc.warm_try(*qp, plain.x, plain.y, added, corrections=8)
  assert r.accepted and r.rounds >= 2


def test_infeasible_problem_is_never_accepted():
  a, b, c, z, p = problems.infeasible(40, 20, 5, 9)
  rng = np.random.default_rng(1)
  for trial in range(3):
    act = rng.uniform(size=40) < 0.3
    r = orc.warm_try(a, b, c, z, p, np.zeros(20), np.zeros(40), act, corrections=3)
    assert not r.accepted


def test_zero_corrections_means_one_round():
  qp, plain, act = _case(17)
  r = orc.warm_try(*qp, np.zeros_like(plain.x), np.zeros_like(plain.y),
                   np.zeros_like(act), corrections=0)
  assert r.rounds == 1


@pytest.mark.parametrize("seed", [3, 11])
def test_ipm_started_from_the_solution_keeps_status_and_is_shorter(seed):
  """The oracle's interior-point method started near the plain solution (y and
  s shifted into the interior by 0.1) ends with the same status and
  objective in fewer iterations than from the cold start."""
  qp, plain, _ = _case(seed)
  a, b, c, z, p = qp
  y0, s0 = plain.y.copy(), plain.s.copy()
  y0[z:] = np.maximum(y0[z:], 0.0) + 0.1
  s0[z:] = np.maximum(s0[z:], 0.0) + 0.1
  s0[:z] = 0.0
  warm = orc.solve(a, b, c, z, p, backend="superlu", init=(plain.x, y0, s0))
  assert warm.status == plain.status
  assert len(warm.stats) < len(plain.stats)
  obj = lambda x: c @ x + 0.5 * x @ (p @ x)
  assert abs(obj(warm.x) - obj(plain.x)) <= 1e-6 * max(1.0, abs(obj(plain.x)))


def test_ipm_start_is_validated():
  qp, plain, _ = _case(3)
  a, b, c, z, p = qp
  with pytest.raises(ValueError, match="positive"):
    orc.solve(a, b, c, z, p, init=(plain.x, np.zeros_like(plain.y), plain.s + 1.0))
  with pytest.raises(ValueError, match="shapes"):
    orc.solve(a, b, c, z, p, init=(plain.x[:-1], plain.y + 1.0, plain.s + 1.0))
