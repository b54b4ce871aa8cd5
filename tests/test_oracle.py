"""Pins the CPU oracle against the reference's own outputs (golden fixtures).

The oracle (oracle/qtqp_oracle.py) is the checker for the CUDA path; these
CPU-only tests prove it reproduces the reference solver: same statuses and
iteration counts, iterates to tight tolerances, and the reference's unit-level
known answers (Ruiz scalings, tau roots, sigma, ratio test).
"""

import numpy as np
import pytest

from oracle import qtqp_oracle as orc
from tests import golden_io

BACKEND = {"SCIPY": "superlu", "SCIPY_DENSE": "dense"}


def _cases():
  out = []
  for name in golden_io.e2e_names():
    for backend in ("SCIPY", "SCIPY_DENSE"):
      for eq in (True, False):
        if golden_io.e2e_result(name, backend, eq) is not None:
          out.append((name, backend, eq))
  return out


@pytest.mark.parametrize("name,backend,eq", _cases())
def test_oracle_matches_reference_solve(name, backend, eq):
  a, b, c, z, p = golden_io.e2e_problem(name)
  ref = golden_io.e2e_result(name, backend, eq)
  got = orc.solve(a, b, c, z, p, backend=BACKEND[backend], equilibrate=eq)
  assert got.status == ref["status"]
  assert len(got.stats) == ref["iters"]
  mus = np.array([st["mu"] for st in got.stats])
  np.testing.assert_allclose(mus, ref["mu"], rtol=1e-6, atol=1e-12)
  if ref["status"] == "solved":  # costs diverge along certificate rays
    pc = np.array([st["pcost"] for st in got.stats])
    np.testing.assert_allclose(pc, ref["pcost"], rtol=1e-7, atol=1e-9)
  # Degenerate problems have non-unique optima; the reference's dsyrk and the
  # oracle's GEMM round differently, so iterates agree to ~1e-6 of their scale.
  for key in ("x", "y", "s"):
    v, r = getattr(got, key), ref[key]
    scale = max(1.0, float(np.nanmax(np.abs(r), initial=0.0)))
    np.testing.assert_allclose(v, r, rtol=1e-5, atol=1e-5 * scale)


@pytest.mark.parametrize("k", range(3))
def test_oracle_ruiz_matches_reference(k):
  d = golden_io.load("reference_units.npz")
  pre = f"ruiz{k}/"
  a, p = golden_io.csc(d, pre + "a"), golden_io.csc(d, pre + "p")
  a_eq, p_eq, _, _, dd, ee = orc.ruiz(a, p, d[pre + "b"], d[pre + "c"])
  # Same elementwise operations in the same order: bit-identical.
  np.testing.assert_array_equal(dd, d[pre + "d"])
  np.testing.assert_array_equal(ee, d[pre + "e"])
  np.testing.assert_array_equal(a_eq.toarray(), d[pre + "a_eq"])
  np.testing.assert_array_equal(p_eq.toarray(), d[pre + "p_eq"])


@pytest.mark.parametrize("k", range(5))
def test_oracle_scalar_kernels_match_reference(k):
  d = golden_io.load("reference_units.npz")
  pre = f"tau{k}/"
  a, p = golden_io.csc(d, pre + "a"), golden_io.csc(d, pre + "p")
  b, c, z = d[pre + "b"], d[pre + "c"], int(d[pre + "z"])
  m, n = a.shape
  q = np.concatenate([c, b])
  mu, sigma = float(d[pre + "mu"]), float(d[pre + "sigma"])
  kq, kr = d[pre + "kinv_q"], d[pre + "kinv_r"]
  ta = float(d[pre + "tau_anchor"])
  tau_q = orc.tau_quadratic(n, q, kq, kr, p, mu, sigma * mu, (mu - sigma * mu) * ta)
  np.testing.assert_allclose(tau_q, d[pre + "tau_quadratic"], rtol=1e-13)
  tau_l = orc.tau_linearized(n, q, kq, kr, p, mu, sigma * mu, d[pre + "x"], d[pre + "y"],
                             0.8, ta)
  np.testing.assert_allclose(tau_l, d[pre + "tau_linearized"], rtol=1e-13)
  y, s = d[pre + "y"], d[pre + "s"]
  sig = orc.sigma_mehrotra(mu, d[pre + "x"], y, float(d[pre + "tau"]), s,
                           float(d[pre + "alpha"]), d[pre + "d_x"], d[pre + "d_y"],
                           float(d[pre + "d_tau"]), d[pre + "d_s"], m, z)
  np.testing.assert_allclose(sig, d[pre + "sigma_out"], rtol=1e-14)
  step = orc.step_size(y, s, d[pre + "d_y"], d[pre + "d_s"], z)
  assert step == float(d[pre + "step"])


def test_oracle_known_answers():
  """README example (x = [0.3, -0.7]) and the minimal QP (x = 1)."""
  import scipy.sparse as sp
  res = orc.solve(sp.csc_matrix([[-1.0, 1.0], [1.0, 0.0], [0.0, 1.0]]),
                  np.array([-1.0, 0.3, -0.5]), np.array([-1.0, -1.0]), 1,
                  sp.csc_matrix([[3.0, -1.0], [-1.0, 2.0]]))
  assert res.status == orc.STATUS_SOLVED
  np.testing.assert_allclose(res.x, [0.3, -0.7], atol=1e-5, rtol=1e-5)
  res = orc.solve(sp.csc_matrix([[-1.0], [1.0]]), np.array([0.0, 2.0]), np.array([-1.0]), 0,
                  sp.csc_matrix([[1.0]]))
  assert res.status == orc.STATUS_SOLVED
  np.testing.assert_allclose(res.x, [1.0], atol=1e-5)


def test_oracle_detects_planted_error():
  """A mistake planted in the oracle's step rule must break parity."""
  a, b, c, z, p = golden_io.e2e_problem("feasible_50x30_s46")
  ref = golden_io.e2e_result("feasible_50x30_s46", "SCIPY_DENSE", True)
  got = orc.solve(a, b, c, z, p, backend="dense", step_size_scale=0.5)
  mus = np.array([st["mu"] for st in got.stats])
  assert len(mus) != ref["iters"] or not np.allclose(mus, ref["mu"], rtol=1e-6)
