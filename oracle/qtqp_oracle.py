"""CPU oracle for the QTQP interior-point hot path (TEST INFRASTRUCTURE ONLY).

This module restates, in plain numpy/scipy, the algorithm of the reference
solver google-deepmind/qtqp v0.0.5 (pure Python).  It exists to check the CUDA
path, never to run inside it: only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py`` (its CPU-baseline leg and ``--impl reference`` arm) may import it.
The product package ``qtqp_b200`` never imports this file.

Parity pin: ``tests/test_oracle.py`` checks this restatement against golden
vectors produced by the reference itself (``tests/golden/make_golden.py``
imports the reference and records its outputs), including the reference's own
known answers (README example x=[0.3,-0.7], the minimal QP x=1).

Each function cites the reference lines it follows (paths relative to the
reference project root).  All arithmetic is FP64, as in the reference.
``warm_try`` restates the device solver's learned-warm-start attempt, which has
no reference counterpart, on the reference's own KKT refinement and
termination test; ``solve(init=...)`` starts the interior-point method from a
given point instead of the reference's cold start (also no counterpart);
``tests/test_oracle_warm.py`` checks both.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EPS = 1e-15  # src/qtqp/__init__.py:51

STATUS_SOLVED = "solved"
STATUS_INFEASIBLE = "infeasible"
STATUS_UNBOUNDED = "unbounded"
STATUS_HIT_MAX_ITER = "hit_max_iter"
STATUS_FAILED = "failed"
STATUS_UNFINISHED = "unfinished"


# ---------------------------------------------------------------------------
# Ruiz equilibration: src/qtqp/__init__.py:616-669
# ---------------------------------------------------------------------------
def ruiz(a: sp.spmatrix, p: sp.spmatrix, b, c, sweeps=10, lo=1e-3, hi=1e3):
  """Returns (a_eq, p_eq, b_eq, c_eq, d, e) with a_eq = D A E, p_eq = E P E.

  Per sweep: row scale 1/sqrt(max|A_row|), column scale
  1/sqrt(max(max|A_col|, max|P_col|)), zero norms replaced by 1, both clipped
  to [lo, hi]; the nonzero a_ij is multiplied by (d_i * e_j)
  (__init__.py:627-651).
  """
  a = sp.csc_matrix(a, dtype=np.float64, copy=True)
  p = sp.csc_matrix(p, dtype=np.float64, copy=True)
  m, n = a.shape
  d = np.ones(m)
  e = np.ones(n)
  for _ in range(sweeps):
    rmax = np.zeros(m)
    if a.nnz:
      np.maximum.at(rmax, a.indices, np.abs(a.data))
    rs = np.clip(1.0 / np.sqrt(np.where(rmax == 0.0, 1.0, rmax)), lo, hi)
    cmax = _col_absmax(a)
    if p.nnz:
      cmax = np.maximum(cmax, _col_absmax(p))
    cs = np.clip(1.0 / np.sqrt(np.where(cmax == 0.0, 1.0, cmax)), lo, hi)
    a.data *= rs[a.indices] * np.repeat(cs, np.diff(a.indptr))
    if p.nnz:
      p.data *= cs[p.indices] * np.repeat(cs, np.diff(p.indptr))
    d *= rs
    e *= cs
  return a, p, b * d, c * e, d, e


def _col_absmax(mat: sp.csc_matrix) -> np.ndarray:
  out = np.zeros(mat.shape[1])
  cnt = np.diff(mat.indptr)
  nzcols = np.nonzero(cnt)[0]
  if len(nzcols):
    out[nzcols] = np.maximum.reduceat(np.abs(mat.data), mat.indptr[nzcols])
  return out


# ---------------------------------------------------------------------------
# KKT backends: the plugin contract of src/qtqp/direct.py:49-109
# ---------------------------------------------------------------------------
class DenseGramKkt:
  """Gram/Schur reduction of the quasi-definite KKT (solvers_dense.py:25-145).

  K = [[P + diag(Rx), A^T], [A, -diag(Ry)]] is solved through
  G = P_off + diag(Rx) + A^T diag(1/Ry) A (+1e-14 max diag G jitter, :112),
  Cholesky (:114), y = (A x - r_y) / Ry (:141).
  """

  def __init__(self, a_eq: sp.spmatrix, p_eq: sp.spmatrix):
    self.a = np.asarray(sp.csr_matrix(a_eq).toarray(), dtype=np.float64)
    pd = np.asarray(sp.csr_matrix(p_eq).toarray(), dtype=np.float64)
    # Symmetric P with its diagonal removed (the diagonal lives in Rx).
    up = np.triu(pd)
    full = up + up.T - np.diag(np.diag(up))
    np.fill_diagonal(full, 0.0)
    self.p_off = full
    self.n = self.a.shape[1]
    self.rx = None
    self.ry = None
    self.chol = None

  def update_diag(self, reg_diag: np.ndarray):
    self.rx = reg_diag[: self.n].copy()
    self.ry = -reg_diag[self.n :]

  def factorize(self):
    g = self.p_off.copy()
    g[np.diag_indices(self.n)] += self.rx
    a_s = self.a * (1.0 / np.sqrt(self.ry))[:, None]
    g += a_s.T @ a_s
    g[np.diag_indices(self.n)] += 1e-14 * np.max(np.diag(g))
    try:
      self.chol = sla.cholesky(g, lower=True)
    except sla.LinAlgError as err:
      raise np.linalg.LinAlgError(f"Cholesky failed: {err}") from err

  def matvec(self, v: np.ndarray) -> np.ndarray:
    n = self.n
    vx, vy = v[:n], v[n:]
    top = self.p_off @ vx + self.rx * vx + self.a.T @ vy
    bot = self.a @ vx - self.ry * vy
    return np.concatenate([top, bot])

  def solve(self, r: np.ndarray) -> np.ndarray:
    n = self.n
    inv_ry = 1.0 / self.ry
    g = r[:n] + self.a.T @ (inv_ry * r[n:])
    x = sla.cho_solve((self.chol, True), g)
    y = inv_ry * (self.a @ x - r[n:])
    return np.concatenate([x, y])


class SuperLUKkt:
  """Full symmetric KKT factorised by SuperLU (solvers_sparse.py:96-121)."""

  def __init__(self, a_eq: sp.spmatrix, p_eq: sp.spmatrix):
    m, n = a_eq.shape
    self.n, self.m = n, m
    p_up = sp.triu(p_eq, format="csc")
    scaffold = sp.bmat(
        [[p_up + sp.eye(n, format="csc"), sp.csc_matrix(a_eq).T],
         [None, sp.eye(m, format="csc")]], format="csc", dtype=np.float64)
    diag = sp.diags(scaffold.diagonal(), format="csc")
    self.full = (scaffold + scaffold.T - diag).tocsc()
    self.full.sort_indices()
    self._didx = _diag_positions(self.full)
    self.lu = None

  def update_diag(self, reg_diag: np.ndarray):
    self.full.data[self._didx] = reg_diag

  def factorize(self):
    self.lu = spla.factorized(self.full)

  def matvec(self, v):
    return self.full @ v

  def solve(self, r):
    return self.lu(r)


def _diag_positions(mat: sp.csc_matrix) -> np.ndarray:
  """Data index of each diagonal entry (direct.py:33-46)."""
  out = np.empty(mat.shape[0], dtype=np.int64)
  for k in range(mat.shape[0]):
    lo, hi = mat.indptr[k], mat.indptr[k + 1]
    out[k] = lo + np.searchsorted(mat.indices[lo:hi], k)
  return out


# ---------------------------------------------------------------------------
# KKT regularisation + iterative refinement: src/qtqp/direct.py:183-307
# ---------------------------------------------------------------------------
class KktIR:
  """Regularised quasi-definite KKT with FP64 iterative refinement."""

  def __init__(self, backend, p_diag, n, m, z, min_reg, max_ir, atol, rtol):
    self.be = backend
    self.p_diag = p_diag
    self.n, self.m, self.z = n, m, z
    self.min_reg, self.max_ir = min_reg, max_ir
    self.atol, self.rtol = atol, rtol
    self.corr = np.zeros(n + m)

  def update(self, mu, s, y):
    """direct.py:183-216: true diag, clamp to min_reg, negate the dual block."""
    n, z = self.n, self.z
    true = np.empty(n + self.m)
    true[:n] = self.p_diag + mu
    true[n:n + z] = mu
    true[n + z:] = s[z:] / y[z:] + mu
    reg = np.maximum(true, self.min_reg)
    true[n:] *= -1.0
    reg[n:] *= -1.0
    self.be.update_diag(reg)
    self.be.factorize()
    self.corr = reg - true

  def solve(self, rhs, warm):
    """direct.py:218-307: refine until ||res||_inf < tol, stall or max_ir."""
    n = self.n
    krhs = rhs.copy()
    krhs[n:] *= -1.0
    rhs_norm = np.linalg.norm(krhs, np.inf)
    tol = self.atol + self.rtol * rhs_norm
    sol = warm.copy()
    res = krhs - self.be.matvec(sol) + self.corr * sol
    rn = np.linalg.norm(res, np.inf)
    status, k = "non-converged", 0
    for k in range(1, self.max_ir + 1):
      prev = rn
      sol = sol + self.be.solve(res)
      res = krhs - self.be.matvec(sol) + self.corr * sol
      rn = np.linalg.norm(res, np.inf)
      if rn < tol:
        status = "converged"
        break
      if rn >= prev:
        status = "stalled"
        break
    if np.any(np.isnan(sol)):
      raise ValueError("Linear solver returned NaNs.")
    return sol, {"solves": k, "final_residual_norm": rn, "rhs_norm": rhs_norm,
                 "tolerance": tol, "converged": status == "converged",
                 "status": status}


# ---------------------------------------------------------------------------
# Scalar kernels of the IPM: src/qtqp/__init__.py:671-886
# ---------------------------------------------------------------------------
def max_step(v, dv):
  """__init__.py:671-680: largest alpha<=1 keeping v + alpha dv >= 0."""
  mask = dv < -EPS
  if not np.any(mask):
    return 1.0
  return min(1.0, float(np.min(-v[mask] / dv[mask])))


def step_size(y, s, dy, ds, z):
  """__init__.py:882-886."""
  return min(max_step(s[z:], ds[z:]), max_step(y[z:], dy[z:]))


def sigma_mehrotra(mu, x, y, tau, s, alpha, dx, dy, dtau, ds, m, z):
  """__init__.py:682-706: sigma = clip((mu_aff/mu)^3, 0, 1), normalised."""
  xa, ya, ta, sa = x + alpha * dx, y + alpha * dy, tau + alpha * dtau, s + alpha * ds
  nrm2 = xa @ xa + ya @ ya + ta * ta
  mu_aff = (m - z + 1) / max(EPS * EPS, nrm2) * (ya @ sa) / (m - z)
  r = mu_aff / max(EPS, mu)
  return float(np.clip(r * r * r, 0.0, 1.0))


def normalize(x, y, tau, s, m, z):
  """__init__.py:859-880: ||(x, y, tau)||^2 = m - z + 1."""
  scale = math.sqrt(m - z + 1) / max(EPS, math.sqrt(x @ x + y @ y + tau * tau))
  return x * scale, y * scale, tau * scale, s * scale


def tau_quadratic(n, q, kq, kr, p_eq, mu, mu_t, r_tau):
  """__init__.py:759-817: root of t_a tau^2 + t_b tau + t_c = 0 (Muller form).

  Raises ValueError for a degenerate equation or a negative/non-finite root.
  """
  ta = mu + kq @ q
  tb = -r_tau - kr @ q
  tc = -mu_t
  if p_eq.nnz > 0:
    pkr = p_eq @ kr[:n]
    pkq = p_eq @ kq[:n]
    ta -= kq[:n] @ pkq
    tb += kr[:n] @ pkq + kq[:n] @ pkr
    tc -= kr[:n] @ pkr
  if abs(ta) < EPS:
    if abs(tb) < EPS:
      raise ValueError("degenerate tau equation")
    root = -tc / tb
    if not np.isfinite(root) or root < -1e-10:
      raise ValueError("invalid linear tau")
    return max(0.0, root)
  disc = tb * tb - 4 * ta * tc
  if disc < -1e-9:
    raise ValueError("negative discriminant")
  disc = max(0.0, disc)
  if tb > 0:
    root = tc / (-0.5 * (tb + math.sqrt(disc)))
  else:
    root = (-0.5 * (tb - math.sqrt(disc))) / ta
  if not np.isfinite(root) or root < -1e-10:
    raise ValueError("invalid tau")
  return max(0.0, root)


def tau_linearized(n, q, kq, kr, p_eq, mu, mu_t, x, y, tau, tau_anchor):
  """__init__.py:819-857: first-order tau update inside [0.1 tau, 10 tau]."""
  px = p_eq @ x if p_eq.nnz > 0 else np.zeros(n)
  qz = q[:n] @ x + q[n:] @ y
  xpx = x @ px
  qkq = q @ kq
  pxkq = px @ kq[:n]
  q_rz = q @ kr - tau * qkq - qz
  px_rz = px @ kr[:n] - tau * pxkq - xpx
  g = mu * tau * tau + (mu_t - mu) * tau_anchor * tau - tau * qz - mu_t - xpx
  num = g - tau * q_rz - 2.0 * px_rz
  den = 2.0 * mu * tau + (mu_t - mu) * tau_anchor - qz + tau * qkq + 2.0 * pxkq
  root = tau + (0.0 if abs(den) < 1e-16 else -num / den)
  if not np.isfinite(root):
    return tau
  return min(max(root, 0.1 * tau), 10.0 * tau)


# ---------------------------------------------------------------------------
# The full solve: src/qtqp/__init__.py:183-307 (validation, presolve) and
# :351-614 (the loop), :888-1008 (termination).
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class OracleResult:
  x: np.ndarray
  y: np.ndarray
  s: np.ndarray
  status: str
  stats: list


def solve(a, b, c, z, p=None, *, atol=1e-7, rtol=1e-8, atol_infeas=1e-8,
          rtol_infeas=1e-9, max_iter=100, step_size_scale=0.99,
          min_static_regularization=1e-8, max_iterative_refinement_steps=20,
          linear_solver_atol=1e-12, linear_solver_rtol=1e-12,
          equilibrate=True, backend="dense", tau_mode="auto", init=None) -> OracleResult:
  """Solves min 1/2 x'Px + c'x s.t. Ax + s = b, s[:z] = 0, s[z:] >= 0.

  backend: "dense" (Gram/Cholesky, solvers_dense.py) or "superlu"
  (solvers_sparse.py:96-121).  tau_mode "linearized" forces the fallback
  (the reference's test_linearized_tau_always_converges patch).  init: an
  optional starting point (x, y, s) in the original scaling that replaces
  _init_variables (no reference counterpart: it restates an interior-point
  method warm-started from a predicted point; s[z:] and y[z:] must be > 0).
  """
  a = sp.csc_matrix(a, dtype=np.float64)
  m_full, n = a.shape
  b = np.array(b, dtype=np.float64)
  c = np.array(c, dtype=np.float64)
  p = sp.csc_matrix((n, n)) if p is None else sp.csc_matrix(p, dtype=np.float64)
  # Presolve (__init__.py:248-270): drop inequality rows with b >= 1e20.
  drop = np.zeros(m_full, dtype=bool)
  drop[z:] = b[z:] >= 1e20
  keep = ~drop
  a_drop, b_drop = a[drop], b[drop]
  a_k, b_k = a[keep], b[keep]
  m = int(keep.sum())
  if z == m:
    raise ValueError("effective z == m after presolve")

  if equilibrate:
    a_eq, p_eq, b_eq, c_eq, d, e = ruiz(a_k, p, b_k, c)
  else:
    a_eq, p_eq, b_eq, c_eq = a_k, p, b_k, c
    d, e = np.ones(m), np.ones(n)
  q = np.concatenate([c_eq, b_eq])
  nb, nc = np.linalg.norm(b_k, np.inf), np.linalg.norm(c, np.inf)

  be = DenseGramKkt(a_eq, p_eq) if backend == "dense" else SuperLUKkt(a_eq, p_eq)
  kkt = KktIR(be, p_eq.diagonal(), n, m, z, min_static_regularization,
              max_iterative_refinement_steps, linear_solver_atol,
              linear_solver_rtol)

  # _init_variables (__init__.py:299-307).
  x = np.zeros(n)
  y = np.zeros(m)
  s = np.zeros(m)
  y[z:] = 1.0
  s[z:] = 1.0
  if init is not None:
    if drop.any():
      raise ValueError("init: problems with rows that the presolve drops are not handled")
    x, y, s = (np.array(v, dtype=np.float64) for v in init)
    if x.shape != (n,) or y.shape != (m,) or s.shape != (m,):
      raise ValueError("init: x, y, s must have the problem's shapes")
    if np.any(y[z:] <= 0.0) or np.any(s[z:] <= 0.0):
      raise ValueError("init: y and s must be positive on the inequality rows")
  x, y, s = x / e, y / d, s * d
  tau = 1.0
  kq = np.zeros(n + m)
  stats = []
  status = STATUS_UNFINISHED
  alpha = sigma = 0.0
  p_nnz = p_eq.nnz

  def newton(mu, mu_t, anchor, tau_anchor, corr_term):
    """__init__.py:708-757."""
    r = (mu - mu_t) * anchor
    if mu_t != 0.0:
      r[n + z:] += mu_t / y[z:]
    r[n + z:] += s[z:]
    if corr_term is not None:
      r[n + z:] += corr_term
    kr, st = kkt.solve(r, anchor)
    tp = None
    if tau_mode != "linearized" and (st["converged"] or
                                     st["final_residual_norm"] < 1e-7):
      try:
        tp = tau_quadratic(n, q, kq, kr, p_eq, mu, mu_t, (mu - mu_t) * tau_anchor)
        st["tau_method"] = "quadratic"
      except ValueError:
        tp = None
    if tp is None:
      st["tau_method"] = "linearized"
      tp = tau_linearized(n, q, kq, kr, p_eq, mu, mu_t, x, y, tau, tau_anchor)
    kr = kr - kq * tp
    return kr[:n].copy(), kr[n:].copy(), tp, st

  it = 0
  for it in range(max_iter):
    st_i: dict[str, Any] = {}
    x, y, tau, s = normalize(x, y, tau, s, m, z)
    mu = (y @ s) / (m - z)
    kkt.update(mu, s, y)
    kq, st_i["q_lin_sys_stats"] = kkt.solve(q, kq)
    xp, yp, tp, st_i["predictor_lin_sys_stats"] = newton(
        mu, 0.0, np.concatenate([x, y]), tau, None)
    dxp, dyp, dtp = xp - x, yp - y, tp - tau
    ds = np.zeros(m)
    ds[z:] = -yp[z:] * s[z:] / y[z:]
    alpha_p = step_size(y, s, dyp, ds, z)
    sigma = sigma_mehrotra(mu, x, y, tau, s, alpha_p, dxp, dyp, dtp, ds, m, z)
    corr_term = -ds[z:] * dyp[z:] / y[z:]
    xc, yc, tc, st_i["corrector_lin_sys_stats"] = newton(
        mu, sigma * mu, np.concatenate([xp, yp]), tp, corr_term)
    dx, dy, dt = xc - x, yc - y, tc - tau
    ds[z:] = sigma * mu / y[z:] + corr_term - yc[z:] * s[z:] / y[z:]
    alpha = step_size(y, s, dy, ds, z)
    stp = step_size_scale * alpha
    x = x + stp * dx
    y = y + stp * dy
    tau = tau + stp * dt
    s = s + stp * ds
    y[z:] = np.maximum(y[z:], 1e-30)
    s[z:] = np.maximum(s[z:], 1e-30)
    tau = max(tau, 1e-30)
    status = _termination(a_k, p, b_k, c, d, e, x, y, tau, s, nb, nc, z,
                          atol, rtol, atol_infeas, rtol_infeas, st_i)
    st_i.update({"iter": it, "mu": mu, "sigma": sigma, "alpha": alpha,
                 "tau": tau})
    stats.append(st_i)
    if status != STATUS_UNFINISHED:
      break
  else:
    status = STATUS_HIT_MAX_ITER
    stats[-1]["status"] = status

  # Finish (__init__.py:580-614) and postsolve (:272-297).
  x, y, s = e * x, d * y, s / d
  if status in (STATUS_SOLVED, STATUS_HIT_MAX_ITER, STATUS_UNFINISHED):
    x, y, s = x / tau, y / tau, s / tau
    y, s = _restore(keep, y, s, 0.0, b_drop - a_drop @ x if drop.any() else 0.0)
    if status == STATUS_UNFINISHED:
      status = STATUS_FAILED
  elif status == STATUS_INFEASIBLE:
    x = np.full(n, np.nan)
    s = np.full(m, np.nan)
    y = y / abs(b_k @ y)
    y, s = _restore(keep, y, s, 0.0, np.nan)
  elif status == STATUS_UNBOUNDED:
    y = np.full(m, np.nan)
    k = abs(c @ x)
    x, s = x / k, s / k
    y, s = _restore(keep, y, s, np.nan, np.nan)
  return OracleResult(x, y, s, status, stats)


def _restore(keep, y, s, y_fill, s_fill):
  if keep.all():
    return y, s
  yf = np.empty(keep.shape[0])
  sf = np.empty(keep.shape[0])
  yf[keep], sf[keep] = y, s
  yf[~keep], sf[~keep] = y_fill, s_fill
  return yf, sf


def _termination(a, p, b, c, d, e, x, y, tau, s, nb, nc, z, atol, rtol,
                 atol_inf, rtol_inf, st):
  """__init__.py:888-990 on the unequilibrated data; fills `st`."""
  x, y, s = e * x, d * y, s / d
  it_ = 1.0 / max(tau, EPS)
  ax = a @ x
  aty = a.T @ y
  px = p @ x if p.nnz else np.zeros(len(x))
  xpx = x @ px if p.nnz else 0.0
  ctx, bty = c @ x, b @ y
  pcost = (ctx + 0.5 * xpx * it_) * it_
  dcost = (-bty - 0.5 * xpx * it_) * it_
  inf = np.inf
  pres = np.linalg.norm((ax + s) * it_ - b, inf)
  dres = np.linalg.norm((px + aty) * it_ + c, inf)
  gap = abs((ctx + bty + xpx * it_) * it_)
  n_aty, n_px = np.linalg.norm(aty, inf), np.linalg.norm(px, inf)
  dinf_a = np.linalg.norm(ax + s, inf) / (abs(ctx) + EPS)
  dinf_p = n_px / (abs(ctx) + EPS)
  dinf = max(dinf_a, dinf_p)
  pinf = n_aty / (abs(bty) + EPS)
  prel = max(np.linalg.norm(ax, inf) * it_, np.linalg.norm(s, inf) * it_, nb)
  drel = max(n_px * it_, n_aty * it_, nc)
  nx, ny = np.linalg.norm(x, inf), np.linalg.norm(y, inf)
  if (gap < atol + rtol * min(abs(pcost), abs(dcost)) and
      pres < atol + rtol * prel and dres < atol + rtol * drel):
    status = STATUS_SOLVED
  elif ctx < -EPS and dinf < atol_inf + rtol_inf * nx / abs(ctx):
    status = STATUS_UNBOUNDED
  elif bty < -EPS and pinf < atol_inf + rtol_inf * ny / abs(bty):
    status = STATUS_INFEASIBLE
  else:
    status = STATUS_UNFINISHED
  st.update({"ctx": ctx, "bty": bty, "pcost": pcost, "dcost": dcost,
             "pres": pres, "dres": dres, "gap": gap, "pinfeas": pinf,
             "dinfeas": dinf, "dinfeas_a": dinf_a, "dinfeas_p": dinf_p,
             "norm_x": nx, "norm_y": ny, "status": status, "prelrhs": prel,
             "drelrhs": drel})
  return status


# ---------------------------------------------------------------------------
# Learned warm start: the reduced KKT attempt (no reference counterpart).
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class WarmResult:
  accepted: bool
  rounds: int        # reduced solves made (1 + corrections used)
  x: np.ndarray      # the last projected point, original scaling
  y: np.ndarray
  s: np.ndarray
  solves: int        # refinement solves over all rounds


def warm_try(a, b, c, z, p, wx, wy, active, *, corrections=0, atol=1e-7, rtol=1e-8,
             atol_infeas=1e-8, rtol_infeas=1e-9, min_static_regularization=1e-8,
             max_iterative_refinement_steps=20, linear_solver_atol=1e-12,
             linear_solver_rtol=1e-12, equilibrate=True, backend="superlu") -> WarmResult:
  """The warm-start attempt of the device solver, restated on the CPU.

  A predicted point (wx, wy; original scaling) and active-row mask decide
  which inequality rows are held tight.  Each round solves the KKT system of
  the equality QP on that set with the reference's regularised factorisation
  and FP64 refinement (direct.py:183-307): true diagonal [diag(P); 0 on tight
  rows, -1e10 on free rows], regularised [max(diag(P), min_reg); -max(min_reg,
  1e-10) on tight rows, -1e10 on free rows], right-hand side -[c; b], warm
  started from the current point.  Then s = b - A x, the point is projected
  onto the cone (y = max(y, 0) on tight rows, y = 0 on free rows, s =
  max(s, 0) on inequality rows, s = 0 on equality rows), and it is accepted
  when the reference's termination test (__init__.py:888-1008) reports
  SOLVED at tau = 1.  Otherwise, while corrections remain, tight rows whose
  dual came out negative leave the set, free rows whose slack came out
  negative enter it, and the next round starts; a round that changes no row
  ends the attempt.  Problems with rows the presolve would drop (b >= 1e20)
  are not handled.
  """
  a = sp.csc_matrix(a, dtype=np.float64)
  m, n = a.shape
  b = np.array(b, dtype=np.float64)
  c = np.array(c, dtype=np.float64)
  p = sp.csc_matrix((n, n)) if p is None else sp.csc_matrix(p, dtype=np.float64)
  if np.any(b[z:] >= 1e20):
    raise ValueError("warm_try: rows that the presolve drops are not handled")
  if equilibrate:
    a_eq, p_eq, b_eq, c_eq, d, e = ruiz(a, p, b, c)
  else:
    a_eq, p_eq, b_eq, c_eq = a, p, b, c
    d, e = np.ones(m), np.ones(n)
  q = np.concatenate([c_eq, b_eq])
  nb, nc = np.linalg.norm(b, np.inf), np.linalg.norm(c, np.inf)
  be = DenseGramKkt(a_eq, p_eq) if backend == "dense" else SuperLUKkt(a_eq, p_eq)
  kkt = KktIR(be, p_eq.diagonal(), n, m, z, min_static_regularization,
              max_iterative_refinement_steps, linear_solver_atol, linear_solver_rtol)
  x = np.asarray(wx, dtype=np.float64) / e
  y = np.asarray(wy, dtype=np.float64) / d
  s = np.zeros(m)
  tight = np.asarray(active, dtype=bool).copy()
  tight[:z] = True
  ineq = np.arange(m) >= z
  dmin, big = max(min_static_regularization, 1e-10), 1e10
  pdiag = p_eq.diagonal()
  true = np.empty(n + m)
  reg = np.empty(n + m)
  true[:n] = pdiag
  reg[:n] = np.maximum(pdiag, min_static_regularization)
  rounds = solves = 0
  for _ in range(1 + max(0, min(corrections, 64))):
    true[n:] = np.where(tight, 0.0, -big)
    reg[n:] = np.where(tight, -dmin, -big)
    be.update_diag(reg)
    try:
      be.factorize()
    except (np.linalg.LinAlgError, RuntimeError):
      break
    kkt.corr = reg - true
    try:
      sol, st = kkt.solve(-q, np.concatenate([x, y]))
    except ValueError:
      break
    rounds += 1
    solves += st["solves"]
    x, ys = sol[:n], sol[n:]
    sk = b_eq - a_eq @ x
    leave = tight & ineq & (ys < 0.0)
    enter = ~tight & ineq & (sk < 0.0)
    y = np.where(ineq, np.where(tight, np.maximum(ys, 0.0), 0.0), ys)
    s = np.where(ineq, np.maximum(sk, 0.0), 0.0)
    status = _termination(a, p, b, c, d, e, x, y, 1.0, s, nb, nc, z, atol, rtol,
                          atol_infeas, rtol_infeas, {})
    if status == STATUS_SOLVED:
      return WarmResult(True, rounds, e * x, d * y, s / d, solves)
    if not (leave.any() or enter.any()):
      break
    tight = (tight & ~leave) | enter
  return WarmResult(False, rounds, e * x, d * y, s / d, solves)
