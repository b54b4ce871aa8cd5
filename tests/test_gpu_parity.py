"""Parity of the CUDA device-resident IPM with the reference (golden fixtures)
and with the oracle, through the public API and the C-ABI.

Criteria (the reference compares backends the same way): identical
SolutionStatus; the solution passes the reference's acceptance conditions;
objective relative error <= 1e-6 against the reference's SCIPY result;
iteration counts equal or within one (reduction order differs).
"""

import numpy as np
import pytest
import scipy.sparse as sp

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import problems
from tests import golden_io, kkt_checks, kkt_driver

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6


def _solve(a, b, c, z, p, **kw):
  kw.setdefault("verbose", False)
  return qb.QTQP(a=a, b=b, c=c, z=z, p=p).solve(linear_solver=qb.LinearSolver.CUDA, **kw)


def _check_against_reference(name, sol, eq=True, backend="SCIPY_DENSE"):
  a, b, c, z, p = golden_io.e2e_problem(name)
  ref = golden_io.e2e_result(name, backend, eq) or golden_io.e2e_result(name, "SCIPY", True)
  assert sol.status.value == ref["status"], (name, sol.status, ref["status"])
  kkt_checks.assert_status_certificate(sol, a, b, c, p, z)
  if ref["status"] == "solved":
    assert kkt_checks.objective_rel_err(sol.x, ref["x"], c, p) <= OBJ_TOL
  return ref


@pytest.mark.parametrize("name", golden_io.e2e_names())
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_ipm_matches_reference(name, precision):
  a, b, c, z, p = golden_io.e2e_problem(name)
  sol = _solve(a, b, c, z, p, collect_stats=True, precision=precision)
  ref = _check_against_reference(name, sol)
  if precision == "fp64":
    assert abs(len(sol.stats) - ref["iters"]) <= 1, (len(sol.stats), ref["iters"])


@pytest.mark.parametrize("name", [n for n in golden_io.e2e_names()
                                  if not n.startswith(("sparse_qp_n200", "small_dense_i"))])
def test_device_ipm_without_equilibration(name):
  a, b, c, z, p = golden_io.e2e_problem(name)
  sol = _solve(a, b, c, z, p, equilibrate=False)
  _check_against_reference(name, sol, eq=False)


def test_fp64_trajectory_follows_reference():
  """Per-iteration mu / sigma / alpha / tau agree with the reference."""
  name = "feasible_150x100_s48"
  a, b, c, z, p = golden_io.e2e_problem(name)
  sol = _solve(a, b, c, z, p, collect_stats=True)
  ref = golden_io.e2e_result(name, "SCIPY_DENSE", True)
  k = min(len(sol.stats), ref["iters"]) - 1
  for key in ("mu", "sigma", "alpha", "tau"):
    got = np.array([st[key] for st in sol.stats[:k]])
    np.testing.assert_allclose(got, ref[key][:k], rtol=1e-5, atol=1e-10, err_msg=key)


def test_batch_matches_oracle_small_dense():
  """64 uneven dense QPs of the batched workload in one launch vs the oracle."""
  qps, refs = [], []
  for i in range(64):
    a, b, c, z, p = problems.small_dense_instance(i)
    qps.append(qb.QTQP(a=a, b=b, c=c, z=z, p=p))
    refs.append(orc.solve(a, b, c, z, p, backend="dense"))
  for precision in ("fp64", "mixed"):
    sols = qb.solve_batch(qps, precision=precision)
    for q, s, r in zip(qps, sols, refs):
      assert s.status.value == r.status
      kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)
      if r.status == "solved":
        assert kkt_checks.objective_rel_err(s.x, r.x, q.c, q.p) <= OBJ_TOL


def test_batch_mixes_statuses():
  """Feasible, infeasible and unbounded QPs in one batch keep their statuses."""
  gens = [problems.feasible(30, 20, 4, 1), problems.infeasible(30, 20, 4, 2),
          problems.unbounded(30, 20, 4, 3), problems.feasible(12, 6, 0, 4)]
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in gens]
  sols = qb.solve_batch(qps)
  assert [s.status.value for s in sols] == ["solved", "infeasible", "unbounded", "solved"]
  for q, s in zip(qps, sols):
    kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)


def test_stats_keys_and_hit_max_iter():
  a, b, c, z, p = golden_io.e2e_problem("feasible_10x5_s42")
  sol = _solve(a, b, c, z, p, collect_stats=True)
  base = {"iter", "pcost", "dcost", "pres", "dres", "gap", "mu", "sigma", "alpha", "tau",
          "norm_x", "norm_y", "status", "time", "prelrhs", "drelrhs", "pinfeas", "dinfeas"}
  extra = {"complementarity", "norm_s", "max_sy", "min_sy", "std_sy", "max_s_over_y",
           "min_s_over_y", "mean_s_over_y", "std_s_over_y"}
  for st in sol.stats:
    assert base <= st.keys() and extra <= st.keys()
  assert [st["iter"] for st in sol.stats] == list(range(len(sol.stats)))
  assert sol.stats[-1]["status"] == qb.SolutionStatus.SOLVED
  assert sol.stats[-1]["complementarity"] < 1e-6
  a, b, c, z, p = golden_io.e2e_problem("feasible_150x100_s48")
  sol = _solve(a, b, c, z, p, max_iter=1, collect_stats=True)
  assert sol.status == qb.SolutionStatus.HIT_MAX_ITER
  assert len(sol.stats) == 1 and sol.stats[0]["status"] == sol.status
  assert np.all(np.isfinite(sol.x)) and np.all(np.isfinite(sol.y))


def test_verbose_output(capsys):
  a, b, c, z, p = golden_io.e2e_problem("readme")
  sol = _solve(a, b, c, z, p, verbose=True)
  out = capsys.readouterr().out
  assert "QTQP" in out and "iter" in out and "Solved" in out
  np.testing.assert_allclose(sol.x, [0.3, -0.7], atol=1e-5, rtol=1e-5)
  _solve(a, b, c, z, p, verbose=False)
  assert capsys.readouterr().out == ""


def test_known_answers_and_edge_shapes():
  sol = _solve(sp.csc_matrix([[-1.0], [1.0]]), np.array([0.0, 2.0]), np.array([-1.0]), 0,
               sp.csc_matrix([[1.0]]))
  np.testing.assert_allclose(sol.x, [1.0], atol=1e-5)
  # LP (p=None) equals explicit zero P (c built for P = 0 so the LP is bounded).
  a, b, c, z, _ = problems.feasible(30, 20, 3, 42, lp=True)
  s1 = qb.QTQP(a=a, b=b, c=c, z=z).solve(verbose=False)
  s2 = qb.QTQP(a=a, b=b, c=c, z=z, p=sp.csc_matrix((20, 20))).solve(verbose=False)
  assert s1.status == s2.status == qb.SolutionStatus.SOLVED
  np.testing.assert_allclose(s1.x, s2.x, atol=1e-8, rtol=1e-8)


@pytest.mark.parametrize("reg", [0.0, 1e-4, 1e-8])
def test_min_static_regularization(reg):
  a, b, c, z, p = problems.feasible(30, 20, 5, 42)
  sol = _solve(a, b, c, z, p, min_static_regularization=reg, max_iterative_refinement_steps=50)
  kkt_checks.assert_solved(sol, a, b, c, p, z)


def test_linearized_tau_mode_converges():
  from qtqp_b200 import batch
  for gen, seed in ((problems.feasible, 1), (problems.infeasible, 2), (problems.unbounded, 3)):
    a, b, c, z, p = gen(60, 40, 5, seed)
    q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
    opts = batch.SolveOptions(tau_mode=1)
    sol = qb.solve_batch([q], _opts=opts)[0]
    kkt_checks.assert_status_certificate(sol, a, b, c, p, z)


def test_plugin_backend_residual():
  """CudaDenseSolver behind DirectKktSolver: KKT residual <= 1e-10
  (the reference's test_direct_linear_solver criterion)."""
  from qtqp_b200 import direct
  for seed in range(3):
    rng = np.random.default_rng(842 + seed)
    m, n, z = 150, 100, 10
    a, b, c, _, p = problems.feasible(m, n, z, rng)
    mu = rng.uniform()
    s = rng.uniform(size=m)
    y = rng.uniform(size=m)
    s[:z] = 0.0
    d = np.concatenate([np.zeros(z), s[z:] / y[z:]])
    for precision in ("fp64", "mixed"):
      kkt = kkt_driver.DirectKktSolver(a=a, p=p, z=z, min_static_regularization=1e-8,
                                   max_iterative_refinement_steps=30, atol=1e-12,
                                   rtol=1e-12, solver=direct.CudaDenseSolver(precision))
      kkt.update(mu=mu, s=s, y=y)
      sol, stats = kkt.solve(rhs=np.concatenate([c, b]), warm_start=np.zeros(n + m))
      kkt.free()
      np.testing.assert_allclose(p @ sol[:n] + mu * sol[:n] + a.T @ sol[n:], c, atol=1e-10,
                                 rtol=1e-10)
      np.testing.assert_allclose(-a @ sol[:n] + (d + mu) * sol[n:], b, atol=1e-10, rtol=1e-10)


def test_plugin_matvec_matches_full_kkt():
  from qtqp_b200 import direct
  rng = np.random.default_rng(2026)
  m, n, z = 20, 12, 4
  a, _, _, _, p = problems.feasible(m, n, z, rng)
  mu = rng.uniform()
  s, y = rng.uniform(size=m), rng.uniform(size=m)
  s[:z] = 0.0
  kkt = kkt_driver.DirectKktSolver(a=a, p=p, z=z, min_static_regularization=1e-8,
                               max_iterative_refinement_steps=2, atol=1e-12, rtol=1e-12,
                               solver=direct.CudaDenseSolver())
  kkt.update(mu=mu, s=s, y=y)
  diag_y = np.full(m, mu)
  diag_y[z:] = s[z:] / y[z:] + mu
  full = sp.bmat([[p + sp.diags(np.full(n, mu)), a.T], [a, -sp.diags(diag_y)]], format="csc")
  vec = rng.normal(size=n + m)
  np.testing.assert_allclose(kkt._solver @ vec, full @ vec, rtol=1e-10, atol=1e-10)


def test_presolve_restores_certificate():
  name = "presolve_infeasible_33x20"
  a, b, c, z, p = golden_io.e2e_problem(name)
  sol = _solve(a, b, c, z, p)
  kkt_checks.assert_infeasible(sol, a, b, z)
  assert sol.y.shape == (33,) and sol.s.shape == (33,)
