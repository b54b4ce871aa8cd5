"""Generates the golden fixtures from the reference solver itself.

Run where a checkout of the reference (google-deepmind/qtqp v0.0.5) is
readable, naming its root in the REFERENCE_ROOT environment variable:

    REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py [e2e] [units]
        [configs] [plugin]

(no names: all four files).  It imports the reference package (pure Python)
under the name ``qtqp_ref`` -- this repository's own package is ``qtqp`` --
together with its test-suite generators, solves a fixed list of seeded problems
with the reference's SCIPY (SuperLU) and SCIPY_DENSE backends, and records
inputs and outputs in tests/golden/*.npz:

  reference_e2e.npz      end-to-end cases (test-suite generators, README, ...)
  reference_units.npz    known answers of hot-path pieces (Ruiz, tau, sigma, ...)
  reference_configs.npz  the benchmark configurations at their stated sizes:
                         the large dense QP (n=4096, m=8192) and 32 held-out
                         instances of the T=50 parametric family
  reference_plugin.npz   the reference's DirectKktSolver (its IR driver) with
                         its dense and SuperLU backends on seeded KKT systems

The tests never import the reference: they read these files.
"""

from __future__ import annotations

import importlib.util
import os
import sys
import warnings

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _load_reference():
  """(qtqp_ref, its tests module).  The reference's modules import each other
  relatively, so the package loads under another name; its test module's
  `import qtqp` is pointed at it."""
  root = os.environ.get("REFERENCE_ROOT")
  if not root:
    raise SystemExit("set REFERENCE_ROOT to the root of a google-deepmind/qtqp v0.0.5 checkout")
  pkg = os.path.join(root, "src", "qtqp")
  spec = importlib.util.spec_from_file_location(
      "qtqp_ref", os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
  qtqp_ref = importlib.util.module_from_spec(spec)
  sys.modules["qtqp_ref"] = qtqp_ref
  spec.loader.exec_module(qtqp_ref)
  sys.modules["qtqp"] = qtqp_ref
  spec = importlib.util.spec_from_file_location(
      "ref_tests", os.path.join(root, "tests", "test_qtqp.py"))
  tests = importlib.util.module_from_spec(spec)
  spec.loader.exec_module(tests)
  return qtqp_ref, tests


def _put_csc(out, prefix, mat):
  mat = sp.csc_matrix(mat)
  mat.sort_indices()
  out[prefix + "_shape"] = np.array(mat.shape)
  out[prefix + "_data"] = mat.data
  out[prefix + "_indices"] = mat.indices.astype(np.int32)
  out[prefix + "_indptr"] = mat.indptr.astype(np.int32)


def _cases(tests):
  """(name, a, b, c, z, p) of every end-to-end case."""
  sys.path.insert(0, REPO)
  from qtqp_b200 import problems  # generators of the benchmark configs
  cases = []

  def add(name, a, b, c, z, p):
    cases.append((name, sp.csc_matrix(a), np.asarray(b, float), np.asarray(c, float), z,
                  sp.csc_matrix(p)))

  for (m, n, z), seeds in (((10, 5, 3), (42, 43)), ((20, 10, 3), (44, 45)),
                           ((50, 30, 5), (46, 47)), ((150, 100, 10), (48,))):
    for s in seeds:
      a, b, c, p = tests._gen_feasible(m, n, z, s)
      add(f"feasible_{m}x{n}_s{s}", a, b, c, z, p)
  for (m, n, z), seeds in (((20, 10, 3), (142, 143)), ((150, 100, 10), (144,))):
    for s in seeds:
      a, b, c, p = tests._gen_infeasible(m, n, z, s)
      add(f"infeasible_{m}x{n}_s{s}", a, b, c, z, p)
  for (m, n, z), seeds in (((20, 10, 3), (242, 243)), ((150, 100, 10), (244,))):
    for s in seeds:
      a, b, c, p = tests._gen_unbounded(m, n, z, s)
      add(f"unbounded_{m}x{n}_s{s}", a, b, c, z, p)
  a, b, c, _ = tests._gen_feasible(50, 30, 5, 4042)
  add("lp_feasible_50x30", a, b, c, 5, sp.csc_matrix((30, 30)))
  a, b, c, p = tests._gen_feasible(50, 30, 0, 4342)
  add("feasible_z0_50x30", a, b, c, 0, p)
  a, b, c, p = tests._gen_feasible(20, 10, 19, 5042)
  add("single_inequality_20x10", a, b, c, 19, p)
  rng = np.random.default_rng(1842)
  a, b, c, p = tests._gen_infeasible(30, 20, 4, rng)
  a2, b2 = tests._append_dropped_inequalities(a, b, 3, rng, 1e21)
  add("presolve_infeasible_33x20", a2, b2, c, 4, p)
  add("readme", [[-1.0, 1.0], [1.0, 0.0], [0.0, 1.0]], [-1.0, 0.3, -0.5], [-1.0, -1.0], 1,
      [[3.0, -1.0], [-1.0, 2.0]])
  add("minimal", [[-1.0], [1.0]], [0.0, 2.0], [-1.0], 0, [[1.0]])
  out = list(cases)
  a, b, c, z, p = problems.sparse_qp_n200()
  out.append(("sparse_qp_n200", a, b, c, z, p))
  for i in range(6):
    a, b, c, z, p = problems.small_dense_instance(i)
    out.append((f"small_dense_i{i}", a, b, c, z, p))
  return out


def make_e2e(qtqp, tests):
  out = {}
  names = []
  for name, a, b, c, z, p in _cases(tests):
    names.append(name)
    _put_csc(out, name + "/a", a)
    _put_csc(out, name + "/p", p)
    out[name + "/b"] = b
    out[name + "/c"] = c
    out[name + "/z"] = np.array(z)
    for backend in ("SCIPY", "SCIPY_DENSE"):
      for eq in (True, False):
        if not eq and (backend == "SCIPY" or name.startswith(("sparse_qp_n200", "small_dense_i"))):
          continue
        tag = f"{name}/{backend}/{'eq' if eq else 'noeq'}"
        sol = qtqp.QTQP(a=a, b=b, c=c, z=z, p=p).solve(
            linear_solver=getattr(qtqp.LinearSolver, backend), verbose=False,
            collect_stats=True, equilibrate=eq)
        out[tag + "/status"] = np.array(sol.status.value)
        out[tag + "/x"] = sol.x
        out[tag + "/y"] = sol.y
        out[tag + "/s"] = sol.s
        out[tag + "/iters"] = np.array(len(sol.stats))
        for key in ("mu", "sigma", "alpha", "tau", "pres", "dres", "gap", "pcost"):
          out[tag + "/" + key] = np.array([st[key] for st in sol.stats])
  out["names"] = np.array(names)
  return out


def make_units(qtqp, tests):
  """Known answers of hot-path pieces, computed by the reference's functions."""
  out = {}
  # Ruiz equilibration (__init__.py:616-663).
  for k, seed in enumerate((2142, 2143, 2144)):
    a, b, c, p = tests._gen_feasible(150, 100, 10, seed)
    solver = qtqp.QTQP(a=a, b=b, c=c, z=10, p=p)
    a_eq, p_eq, b_eq, c_eq, d, e = solver._equilibrate()
    pre = f"ruiz{k}/"
    _put_csc(out, pre + "a", a)
    _put_csc(out, pre + "p", p)
    out[pre + "b"], out[pre + "c"] = b, c
    out[pre + "d"], out[pre + "e"] = d, e
    out[pre + "a_eq"] = a_eq.toarray()
    out[pre + "p_eq"] = p_eq.toarray()
  # Quadratic / linearised tau, sigma, step size on random data.
  rng = np.random.default_rng(1142)
  for k in range(5):
    m, n, z = 150, 100, 10
    a, b, c, p = tests._gen_feasible(m, n, z, int(rng.integers(1 << 30)))
    mu = rng.uniform()
    sigma = rng.uniform()
    s = rng.uniform(size=m)
    y = rng.uniform(size=m)
    s[:z] = 0.0
    solver = qtqp.QTQP(a=a, b=b, c=c, z=z, p=p)
    solver.q = np.concatenate([c, b])
    kkt = qtqp.direct.DirectKktSolver(
        a=a, p=p, z=z, min_static_regularization=1e-8, max_iterative_refinement_steps=10,
        atol=1e-12, rtol=1e-12, solver=qtqp.direct.ScipySolver())
    kkt.update(mu=mu, s=s, y=y)
    solver.kinv_q, _ = kkt.solve(rhs=solver.q, warm_start=np.zeros(n + m))
    r_anchor = rng.uniform(size=n + m)
    r = (mu - sigma * mu) * r_anchor
    r[n + z:] += sigma * mu / y[z:] + s[z:]
    kinv_r, _ = kkt.solve(rhs=r, warm_start=np.zeros(n + m))
    tau_anchor = rng.uniform()
    x = rng.normal(size=n)
    pre = f"tau{k}/"
    _put_csc(out, pre + "a", a)
    _put_csc(out, pre + "p", p)
    out[pre + "b"], out[pre + "c"], out[pre + "z"] = b, c, np.array(z)
    out[pre + "mu"], out[pre + "sigma"] = np.array(mu), np.array(sigma)
    out[pre + "s"], out[pre + "y"], out[pre + "r"] = s, y, r
    out[pre + "kinv_q"], out[pre + "kinv_r"] = solver.kinv_q, kinv_r
    out[pre + "tau_anchor"], out[pre + "x"] = np.array(tau_anchor), x
    out[pre + "tau_quadratic"] = np.array(solver._solve_for_tau(
        p, kinv_r, mu, sigma * mu, (mu - sigma * mu) * tau_anchor))
    out[pre + "tau_linearized"] = np.array(solver._solve_for_tau_linearized_fallback(
        p, kinv_r, mu, sigma * mu, x, y, 0.8, tau_anchor))
    alpha = rng.uniform()
    d_x, d_y, d_s = rng.normal(size=n), rng.normal(size=m), rng.normal(size=m)
    d_tau = rng.normal()
    tau = rng.uniform(0.1, 2.0)
    out[pre + "alpha"], out[pre + "tau"], out[pre + "d_tau"] = (
        np.array(alpha), np.array(tau), np.array(d_tau))
    out[pre + "d_x"], out[pre + "d_y"], out[pre + "d_s"] = d_x, d_y, d_s
    out[pre + "sigma_out"] = np.array(solver._compute_sigma(
        mu, x, y, tau, s, alpha, d_x, d_y, d_tau, d_s))
    out[pre + "step"] = np.array(solver._compute_step_size(y, s, d_y, d_s))
  return out


def _objective(a, b, c, p, x):
  return float(c @ x + 0.5 * x @ (p @ x))


PARAM_TEST_FIRST = 16384  # held-out split of the 20000-instance family
PARAM_CASES = 32


def make_configs(qtqp):
  """The large dense QP and held-out parametric instances at full size:
  status, iterations, objective (and x for the large QP)."""
  sys.path.insert(0, REPO)
  from qtqp_b200 import problems
  out = {}
  a, b, c, z, p = problems.large_dense()
  a, p = sp.csc_matrix(a), sp.csc_matrix(p)
  sol = qtqp.QTQP(a=a, b=b, c=c, z=z, p=p).solve(
      linear_solver=qtqp.LinearSolver.SCIPY_DENSE, verbose=False, collect_stats=True)
  out["large_dense/status"] = np.array(sol.status.value)
  out["large_dense/iters"] = np.array(len(sol.stats))
  out["large_dense/objective"] = np.array(_objective(a, b, c, p, sol.x))
  out["large_dense/x"] = sol.x
  out["large_dense/mu"] = np.array([st["mu"] for st in sol.stats])
  fam = problems.parametric_mpc_family()
  idx = np.arange(PARAM_TEST_FIRST, PARAM_TEST_FIRST + PARAM_CASES)
  status, iters, obj = [], [], []
  for i in idx:
    a, b, c, z, p = problems.parametric_mpc_instance(fam, int(i))
    a, p = sp.csc_matrix(a), sp.csc_matrix(p)
    sol = qtqp.QTQP(a=a, b=b, c=c, z=z, p=p).solve(
        linear_solver=qtqp.LinearSolver.SCIPY, verbose=False, collect_stats=True)
    status.append(sol.status.value)
    iters.append(len(sol.stats))
    obj.append(_objective(a, b, c, p, sol.x) if sol.status.value == "solved" else np.nan)
  out["parametric/index"] = idx
  out["parametric/status"] = np.array(status)
  out["parametric/iters"] = np.array(iters)
  out["parametric/objective"] = np.array(obj)
  return out


def make_plugin(qtqp, tests):
  """The reference's DirectKktSolver driving its dense (SCIPY_DENSE) and
  SuperLU (SCIPY) backends on seeded regularised KKT systems: the solution,
  the refinement statistics, and the inputs that produced them."""
  out = {}
  rng = np.random.default_rng(3142)
  for k in range(4):
    m, n, z = (150, 100, 10) if k < 3 else (40, 25, 5)
    a, b, c, p = tests._gen_feasible(m, n, z, int(rng.integers(1 << 30)))
    mu = float(rng.uniform(1e-6, 1.0))
    s = rng.uniform(size=m)
    y = rng.uniform(size=m)
    s[:z] = 0.0
    rhs = rng.normal(size=n + m)
    pre = f"plugin{k}/"
    _put_csc(out, pre + "a", a)
    _put_csc(out, pre + "p", p)
    out[pre + "z"], out[pre + "mu"] = np.array(z), np.array(mu)
    out[pre + "s"], out[pre + "y"], out[pre + "rhs"] = s, y, rhs
    for backend, cls in (("dense", qtqp.direct.ScipyDenseSolver),
                         ("superlu", qtqp.direct.ScipySolver)):
      kkt = qtqp.direct.DirectKktSolver(
          a=a, p=p, z=z, min_static_regularization=1e-8, max_iterative_refinement_steps=20,
          atol=1e-12, rtol=1e-12, solver=cls())
      kkt.update(mu=mu, s=s, y=y)
      sol, st = kkt.solve(rhs=rhs, warm_start=np.zeros(n + m))
      kkt.free()
      out[pre + backend + "/sol"] = sol
      out[pre + backend + "/solves"] = np.array(st["solves"])
      out[pre + backend + "/final_residual_norm"] = np.array(st["final_residual_norm"])
      out[pre + backend + "/status"] = np.array(st["status"])
  return out


def main():
  warnings.simplefilter("ignore")
  which = set(sys.argv[1:]) or {"e2e", "units", "configs", "plugin"}
  qtqp, tests = _load_reference()
  if "e2e" in which:
    np.savez_compressed(os.path.join(HERE, "reference_e2e.npz"), **make_e2e(qtqp, tests))
  if "units" in which:
    np.savez_compressed(os.path.join(HERE, "reference_units.npz"), **make_units(qtqp, tests))
  if "configs" in which:
    np.savez_compressed(os.path.join(HERE, "reference_configs.npz"), **make_configs(qtqp))
  if "plugin" in which:
    np.savez_compressed(os.path.join(HERE, "reference_plugin.npz"), **make_plugin(qtqp, tests))
  print("wrote", sorted(which))


if __name__ == "__main__":
  main()
