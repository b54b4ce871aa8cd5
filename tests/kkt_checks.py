"""Acceptance criteria for a returned Solution.

These are the reference suite's acceptance conditions (tests/test_qtqp.py,
_assert_solution / _assert_infeasible / _assert_unbounded), written as plain
functions: relative duality gap, primal and dual residuals within atol+rtol
scaled tolerances and cone feasibility for SOLVED; b'y = -1 with A'y ~ 0 for
INFEASIBLE; c'x = -1 with Ax + s ~ 0, Px ~ 0 for UNBOUNDED.
"""

import numpy as np


def kkt_errors(x, y, s, a, b, c, p):
  px = p @ x
  pcost = c @ x + 0.5 * x @ px
  dcost = -b @ y - 0.5 * x @ px
  ax, aty = a @ x, a.T @ y
  inf = np.inf
  return dict(
      pcost=pcost, dcost=dcost,
      gap=abs(c @ x + b @ y + x @ px),
      pres=np.linalg.norm(ax + s - b, inf),
      dres=np.linalg.norm(px + aty + c, inf),
      prel=max(np.linalg.norm(ax, inf), np.linalg.norm(s, inf), np.linalg.norm(b, inf)),
      drel=max(np.linalg.norm(px, inf), np.linalg.norm(aty, inf), np.linalg.norm(c, inf)))


def assert_solved(sol, a, b, c, p, z, atol=1e-7, rtol=1e-8):
  assert sol.status.value == "solved", sol.status
  e = kkt_errors(sol.x, sol.y, sol.s, a, b, c, p)
  assert e["gap"] < atol + rtol * min(abs(e["pcost"]), abs(e["dcost"])), e
  assert e["pres"] < atol + rtol * e["prel"], e
  assert e["dres"] < atol + rtol * e["drel"], e
  assert np.min(sol.y[z:], initial=0.0) > -1e-9
  assert np.min(sol.s[z:], initial=0.0) > -1e-9


def assert_infeasible(sol, a, b, z, atol=1e-8, rtol=1e-9):
  assert sol.status.value == "infeasible", sol.status
  assert np.all(np.isnan(sol.x)) and np.all(np.isnan(sol.s))
  np.testing.assert_allclose(b @ sol.y, -1.0, atol=atol, rtol=rtol)
  assert np.min(sol.y[z:], initial=0.0) > -1e-9
  assert np.linalg.norm(a.T @ sol.y, np.inf) < atol + rtol * np.linalg.norm(sol.y, np.inf)


def assert_unbounded(sol, a, c, p, z, atol=1e-8, rtol=1e-9):
  assert sol.status.value == "unbounded", sol.status
  assert np.all(np.isnan(sol.y))
  np.testing.assert_allclose(c @ sol.x, -1.0, atol=atol, rtol=rtol)
  m = a.shape[0]
  assert np.min(sol.s[z:m], initial=0.0) > -1e-9
  nx = np.linalg.norm(sol.x, np.inf)
  assert np.linalg.norm(a @ sol.x + sol.s[:m], np.inf) < atol + rtol * nx
  assert np.linalg.norm(p @ sol.x, np.inf) < atol + rtol * nx


def assert_status_certificate(sol, a, b, c, p, z):
  st = sol.status.value
  if st == "solved":
    assert_solved(sol, a, b, c, p, z)
  elif st == "infeasible":
    assert_infeasible(sol, a, b, z)
  elif st == "unbounded":
    assert_unbounded(sol, a, c, p, z)
  else:
    raise AssertionError(f"unexpected status {st}")


def objective_rel_err(x, x_ref, c, p):
  f = c @ x + 0.5 * x @ (p @ x)
  f_ref = c @ x_ref + 0.5 * x_ref @ (p @ x_ref)
  return abs(f - f_ref) / max(1.0, abs(f_ref))
