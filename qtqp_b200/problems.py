"""Seeded synthetic QP generators.

Workloads: the five benchmark configurations (a single sparse QP, a batch of
uneven small dense QPs, a large dense QP, a long-horizon MPC QP and its
parametric family) and the three certificate families used by the tests
(feasible, primal infeasible, dual infeasible).  Every generator takes a seed
and returns (a: csc, b, c, z, p: csc).

Seeds: the single sparse QP uses ``default_rng(1000)``, the small dense batch
1001, the large dense QP 1002, the MPC QP 1003 and the parametric family 1004;
instance i of a batch uses ``default_rng([base, i])``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _feasible_pair(rng, a, p, z):
  """b, c from a primal-dual optimal pair (x0, y0, s0).

  x0 ~ N(0,1); y0[:z] ~ N(0,1); y0[z:] = |N(0,1)| on a random half, else 0;
  s0[:z] = 0; s0[z:] ~ U(0,1) where y0 == 0, else 0 (complementary).
  """
  m, n = a.shape
  x0 = rng.normal(size=n)
  y0 = np.zeros(m)
  y0[:z] = rng.normal(size=z)
  active = rng.random(m - z) < 0.5
  y0[z:] = np.where(active, np.abs(rng.normal(size=m - z)), 0.0)
  s0 = np.zeros(m)
  s0[z:] = np.where(active, 0.0, rng.random(m - z))
  b = a @ x0 + s0
  c = -(p @ x0 + a.T @ y0)
  return np.asarray(b).ravel(), np.asarray(c).ravel()


# ---------------------------------------------------------------------------
# Benchmark configurations.
# ---------------------------------------------------------------------------
SPARSE_QP_M_DENSITY = 0.10  # density of M in P = M M^T + 1e-2 I (not fixed upstream)


def sparse_qp_n200(seed: int = 1000):
  """Single sparse QP: n=200, m=300, z=50; A = 5% Bernoulli mask x N(0,1);
  P = M M^T + 1e-2 I with M 200x20 sparse N(0,1) (10% dense)."""
  rng = np.random.default_rng(seed)
  n, m, z = 200, 300, 50
  mask = rng.random((m, n)) < 0.05
  a = sp.csc_matrix(np.where(mask, rng.normal(size=(m, n)), 0.0))
  mm = sp.random(n, 20, density=SPARSE_QP_M_DENSITY, format="csc", rng=rng,
                 data_rvs=lambda k: rng.normal(size=k))
  p = sp.csc_matrix(mm @ mm.T + 1e-2 * sp.eye(n))
  b, c = _feasible_pair(rng, a, p, z)
  return a, b, c, z, p


def small_dense_instance(i: int, base: int = 1001):
  """One of the uneven small dense QPs: n ~ U{8..64}, m = 2n, z = n // 4,
  A ~ N(0,1) dense, P = L L^T + 1e-3 I with L n x n//2 ~ N(0,1)."""
  rng = np.random.default_rng([base, i])
  n = int(rng.integers(8, 65))
  m, z = 2 * n, n // 4
  a_d = rng.normal(size=(m, n))
  l = rng.normal(size=(n, n // 2))
  p_d = l @ l.T + 1e-3 * np.eye(n)
  p_d = 0.5 * (p_d + p_d.T)
  b, c = _feasible_pair(rng, a_d, p_d, z)
  return sp.csc_matrix(a_d), b, c, z, sp.csc_matrix(p_d)


def small_dense_instance_n(n: int, i: int, base: int = 7):
  """Like small_dense_instance, with n fixed (m = 2n, z = n // 4): batches of
  one size, for per-size timing of the batch kernel."""
  rng = np.random.default_rng([base, n, i])
  m, z = 2 * n, n // 4
  a_d = rng.normal(size=(m, n))
  l = rng.normal(size=(n, n // 2))
  p_d = l @ l.T + 1e-3 * np.eye(n)
  p_d = 0.5 * (p_d + p_d.T)
  b, c = _feasible_pair(rng, a_d, p_d, z)
  return sp.csc_matrix(a_d), b, c, z, sp.csc_matrix(p_d)


def small_dense_size(i: int, base: int = 1001) -> tuple[int, int]:
  """(n, m) of small_dense_instance(i) without building it (the same first
  draw of the same generator)."""
  n = int(np.random.default_rng([base, i]).integers(8, 65))
  return n, 2 * n


def small_dense_batch(count: int = 4096):
  return [small_dense_instance(i) for i in range(count)]


def large_dense(seed: int = 1002, n: int = 4096, m: int = 8192, z: int = 1024, rank: int = 256):
  """Large dense QP: A ~ N(0, 1/n); P = U diag(d) U^T + 1e-4 I with U n x rank
  ~ N(0,1), d ~ U(0.1, 10).  Returns dense arrays (a, b, c, z, p)."""
  rng = np.random.default_rng(seed)
  a = rng.normal(scale=1.0 / np.sqrt(n), size=(m, n))
  u = rng.normal(size=(n, rank))
  d = rng.uniform(0.1, 10.0, size=rank)
  p = (u * d) @ u.T + 1e-4 * np.eye(n)
  p = 0.5 * (p + p.T)
  b, c = _feasible_pair(rng, a, p, z)
  return a, b, c, z, p


def mpc_structure(horizon: int, nx: int = 40, nu: int = 20, seed: int = 1003):
  """Stage-interleaved MPC QP structure [x_0, u_0, ..., x_{T-1}, u_{T-1}]:
  equalities x_0 = b_0, x_{t+1} - A_d x_t - B_d u_t = b_t; box rows [I; -I]
  with bounds 5 (x) and 1 (u); P = blockdiag(diag(Q), 0.1 I).
  Returns (a csc, z, p csc, ub)."""
  rng = np.random.default_rng(seed)
  st = nx + nu
  n = horizon * st
  ad = np.eye(nx) + 0.01 * rng.normal(size=(nx, nx))
  bd = rng.normal(scale=1.0 / np.sqrt(nx), size=(nx, nu))
  rows, cols, vals = [], [], []
  for k in range(nx):  # x_0 = b_0
    rows.append(k)
    cols.append(k)
    vals.append(1.0)
  r0 = nx
  for t in range(horizon - 1):
    xt, ut, xn = t * st, t * st + nx, (t + 1) * st
    for i in range(nx):
      rows.append(r0 + i)
      cols.append(xn + i)
      vals.append(1.0)
      for j in range(nx):
        rows.append(r0 + i)
        cols.append(xt + j)
        vals.append(-ad[i, j])
      for j in range(nu):
        rows.append(r0 + i)
        cols.append(ut + j)
        vals.append(-bd[i, j])
    r0 += nx
  z = r0
  a_eq = sp.csc_matrix((vals, (rows, cols)), shape=(z, n))
  eye = sp.eye(n, format="csc")
  a = sp.vstack([a_eq, eye, -eye], format="csc")
  q = rng.uniform(0.1, 1.0, size=nx)
  pdiag = np.tile(np.concatenate([q, np.full(nu, 0.1)]), horizon)
  p = sp.diags(pdiag, format="csc")
  ub = np.tile(np.concatenate([np.full(nx, 5.0), np.full(nu, 1.0)]), horizon)
  return a, z, p, ub


def mpc_feasible(horizon: int, seed: int = 1003, active_frac: float = 0.1,
                 free_initial: bool = False, nx: int = 40, nu: int = 20):
  """MPC QP with b, c from a feasible pair: x_bar strictly inside the boxes
  except a fraction `active_frac` at +-bound (with positive duals there).
  free_initial keeps the first stage's variables off the bounds."""
  a, z, p, ub = mpc_structure(horizon, nx=nx, nu=nu, seed=seed)
  rng = np.random.default_rng([seed, 1])
  n = p.shape[0]
  xbar = rng.uniform(-0.5, 0.5, size=n) * ub
  act = rng.random(n) < active_frac
  if free_initial:
    act[:60] = False
  sgn = np.where(rng.random(n) < 0.5, 1.0, -1.0)
  xbar = np.where(act, sgn * ub, xbar)
  ybar = np.zeros(a.shape[0])
  ybar[:z] = rng.normal(size=z)
  lam = np.abs(rng.normal(size=n))
  ybar[z:z + n] = np.where(act & (sgn > 0), lam, 0.0)       # x <= ub active
  ybar[z + n:] = np.where(act & (sgn < 0), lam, 0.0)        # -x <= ub active
  b = np.concatenate([a[:z] @ xbar, ub, ub])
  c = -(p @ xbar + a.T @ ybar)
  return a, b, c, z, p


def mpc_t500():
  return mpc_feasible(500)


PARAMETRIC_NX = 40  # initial-state rows of b carry the parameter


def parametric_mpc_family(count: int = 20000, horizon: int = 50, dim: int = 32, seed: int = 1004):
  """Parametric family: fixed (A, P) of the T=50 MPC QP; (b, c) = (b_bar,
  c_bar) + W theta, theta ~ N(0, I_dim), W with N(0, 0.1^2) entries (std 0.1).

  W is non-zero on the rows of b that fix the initial state (the first nx
  equality rows) and on every entry of c; its rows for the dynamics offsets
  and the box bounds are zero.  Perturbing those as well makes almost every
  instance infeasible (2045 of 2048 measured): the state is pinned at t=0 and
  random dynamics offsets drift it out of the |x| <= 5 box faster than the
  |u| <= 1 inputs can steer.  The base point keeps the initial state inside
  the box.  Returns (a, z, p, b_bar, c_bar, W, thetas).
  """
  a, b_bar, c_bar, z, p = mpc_feasible(horizon, seed=seed, free_initial=True)
  rng = np.random.default_rng(seed)
  mtot, n = a.shape
  w = np.zeros((mtot + n, dim))
  w[:PARAMETRIC_NX] = rng.normal(scale=0.1, size=(PARAMETRIC_NX, dim))
  w[mtot:] = rng.normal(scale=0.1, size=(n, dim))
  thetas = np.random.default_rng([seed, 2]).normal(size=(count, dim))
  return a, z, p, b_bar, c_bar, w, thetas


def parametric_mpc_instance(family, i: int):
  """(a, b, c, z, p) of instance i of a family from parametric_mpc_family."""
  a, z, p, b_bar, c_bar, w, thetas = family
  d = w @ thetas[i]
  m = a.shape[0]
  return a, b_bar + d[:m], c_bar + d[m:], z, p


# ---------------------------------------------------------------------------
# Certificate families for tests.
# ---------------------------------------------------------------------------
def feasible(m: int, n: int, z: int, seed, density: float = 0.1, lp: bool = False):
  """Sparse feasible QP with a known optimal primal-dual pair (P = 0 if lp)."""
  rng = np.random.default_rng(seed)
  a = sp.random(m, n, density=density, format="csc", rng=rng,
                data_rvs=lambda k: rng.normal(size=k))
  g = sp.random(n, n, density=0.05, format="csc", rng=rng,
                data_rvs=lambda k: rng.normal(size=k))
  p = sp.csc_matrix((n, n)) if lp else sp.csc_matrix(0.01 * (g.T @ g))
  b, c = _feasible_pair(rng, a, p, z)
  return a, b, c, z, p


def infeasible(m: int, n: int, z: int, seed):
  """Primal infeasible QP: a Farkas ray y (y[z:] >= 0, A^T y = 0, b^T y = -1)."""
  rng = np.random.default_rng(seed)
  y = rng.random(m) + 0.1
  a = rng.normal(size=(m, n))
  a -= np.outer(y, y @ a) / (y @ y)
  b = rng.normal(size=m)
  b = -b / (b @ y)
  g = rng.normal(size=(n, n))
  p = 0.01 * g.T @ g
  c = rng.normal(size=n)
  return sp.csc_matrix(a), b, c, z, sp.csc_matrix(p)


def unbounded(m: int, n: int, z: int, seed):
  """Dual infeasible QP: a ray x with P x = 0, A x + s = 0 (s[z:] >= 0,
  s[:z] = 0) and c^T x = -1."""
  rng = np.random.default_rng(seed)
  g = rng.normal(size=(n, n))
  p = 0.01 * g.T @ g
  w, v = np.linalg.eigh(p)
  w[0] = 0.0
  p = (v * w) @ v.T
  p = 0.5 * (p + p.T)
  x = v[:, 0]
  s = np.zeros(m)
  s[z:] = rng.random(m - z)
  a = rng.normal(size=(m, n))
  a -= np.outer(a @ x + s, x) / (x @ x)
  c = rng.normal(size=n)
  c = -c / (c @ x)
  b = rng.normal(size=m)
  return sp.csc_matrix(a), b, c, z, sp.csc_matrix(p)


# ---------------------------------------------------------------------------
# Sparse QPs whose Gram matrix is neither dense nor banded (the supernodal
# path): random sparse rows, and min-cost flows on a grid network.
# ---------------------------------------------------------------------------
def sparse_rows(m: int, n: int, per_row: int, rng) -> sp.csc_matrix:
  """m x n, each row with `per_row` N(0,1) entries in random columns (every
  column hit at least once)."""
  cols = np.concatenate([rng.permutation(n), rng.integers(0, n, size=m * per_row - n)])
  cols = cols[:m * per_row] if m * per_row >= n else cols
  rows = np.repeat(np.arange(m), per_row)[:cols.size]
  a = sp.csc_matrix((rng.normal(size=cols.size), (rows, cols)), shape=(m, n))
  a.sum_duplicates()
  return a


def sparse_feasible(n: int, m: int, z: int, seed, per_row: int = 3, lp: bool = False):
  """Sparse feasible QP: A with `per_row` entries per row, P = 0.1 G^T G + 1e-2 I
  with G two entries per row (P = 0 if lp), b and c from a known optimal pair."""
  rng = np.random.default_rng(seed)
  a = sparse_rows(m, n, per_row, rng)
  if lp:
    p = sp.csc_matrix((n, n))
  else:
    g = sparse_rows(n, n, 2, rng)
    p = sp.csc_matrix(0.1 * (g.T @ g) + 1e-2 * sp.eye(n))
  b, c = _feasible_pair(rng, a, p, z)
  return a, b, c, z, p


def sparse_infeasible(n: int, m: int, z: int, seed, per_row: int = 3):
  """Sparse primal-infeasible QP: two inequality rows a x <= b1, -a x <= b2
  with b1 + b2 = -1 (the Farkas ray y = e_i + e_j)."""
  a, b, c, z, p = sparse_feasible(n, m, z, seed, per_row)
  a = sp.lil_matrix(a)
  i, j = m - 2, m - 1
  a[j, :] = -a[i, :]
  b = b.copy()
  b[j] = -1.0 - b[i]
  return sp.csc_matrix(a), b, c, z, p


def sparse_unbounded(n: int, m: int, z: int, seed, per_row: int = 3):
  """Sparse dual-infeasible QP: variable k has no entry in P or in the
  equality rows, entries <= 0 in the inequality rows, and c_k = -1, so
  x = t e_k stays feasible with the objective going to -inf."""
  rng = np.random.default_rng(seed)
  a, b, c, z, p = sparse_feasible(n, m, z, seed, per_row)
  k = n - 1
  a = sp.lil_matrix(a)
  col = a[:, k].toarray().ravel()
  col[:z] = 0.0
  col[z:] = -np.abs(col[z:])
  a[:, k] = col.reshape(-1, 1)
  p = sp.lil_matrix(p)
  p[k, :] = 0.0
  p[:, k] = 0.0
  c = c.copy()
  c[k] = -1.0
  b = b + rng.random(m)  # keeps the QP feasible (x0 with slack)
  return sp.csc_matrix(a), b, c, z, sp.csc_matrix(p)


def grid_flow(k: int, seed: int = 1005):
  """Min-cost flow with quadratic edge costs on a k x k grid network (both
  directions of every grid edge): node conservation E x = d (equalities) and
  0 <= x <= u (inequalities), from a known optimal pair.  n = 4 k (k - 1)."""
  rng = np.random.default_rng(seed)
  idx = np.arange(k * k).reshape(k, k)
  e = ([(idx[i, j], idx[i, j + 1]) for i in range(k) for j in range(k - 1)] +
       [(idx[i, j], idx[i + 1, j]) for i in range(k - 1) for j in range(k)])
  e = e + [(v, u) for u, v in e]
  n, nodes = len(e), k * k
  tail = np.array([u for u, _ in e])
  head = np.array([v for _, v in e])
  inc = sp.csc_matrix((np.concatenate([-np.ones(n), np.ones(n)]),
                       (np.concatenate([tail, head]), np.tile(np.arange(n), 2))),
                      shape=(nodes, n))
  eye = sp.eye(n, format="csc")
  a = sp.csc_matrix(sp.vstack([inc, -eye, eye]))
  p = sp.csc_matrix(sp.diags(rng.uniform(0.1, 1.0, size=n)))
  b, c = _feasible_pair(rng, a, p, nodes)
  return a, b, c, nodes, p
