"""Host-side KKT refinement driver used by the tests to exercise a plugin.

A restatement of the reference's ``DirectKktSolver`` (src/qtqp/direct.py:
112-311): the regularised diagonal and its correction (update, :183-216) and
the FP64 iterative refinement with its stall rule and NaN check (solve,
:218-307), with the same buffers and stats keys.  The library's device loop
does not use it (it has its own refinement, ``Ipm::ir_solve``); it is test
infrastructure that runs a ``direct.LinearSolver`` backend the way the
reference's host loop does.
"""

from __future__ import annotations

import logging
from typing import Any

import numpy as np
import scipy.sparse as sp

from qtqp_b200.direct import LinearSolver


class DirectKktSolver:
  """Regularised KKT solve with FP64 iterative refinement (direct.py:112-311).

      [ P + mu I        A^T      ] [x]   [ rhs_x ]
      [     A      -(D + mu I)   ] [y] = [-rhs_y ]
  """

  def __init__(self, *, a, p, z, min_static_regularization,
               max_iterative_refinement_steps, atol, rtol, solver: LinearSolver):
    self.m, self.n = a.shape
    self.z = z
    self._p_diags = p.diagonal()
    self.min_static_regularization = min_static_regularization
    self.max_iterative_refinement_steps = max_iterative_refinement_steps
    self._atol, self._rtol = atol, rtol
    self._solver = solver
    solver.set_dims(n=self.n, m=self.m, z=self.z)
    self._kkt = sp.bmat(
        [[sp.triu(p, format="csc") + sp.eye(self.n, format="csc"), a.T],
         [None, sp.eye(self.m, format="csc")]],
        format=solver.format(), dtype=np.float64)
    solver.set_kkt(self._kkt)
    nm = self.n + self.m
    self._true = np.empty(nm)
    self._reg = np.empty(nm)
    self._rhs = np.empty(nm)
    self._corr = np.zeros(nm)

  def update(self, mu: float, s: np.ndarray, y: np.ndarray) -> None:
    n, z = self.n, self.z
    self._true[:n] = self._p_diags
    self._true[:n] += mu
    self._true[n:n + z] = mu
    self._true[n + z:] = s[z:] / y[z:] + mu
    np.maximum(self._true, self.min_static_regularization, out=self._reg)
    self._true[n:] *= -1.0
    self._reg[n:] *= -1.0
    self._solver.update_diag(self._reg)
    self._solver.factorize()
    np.subtract(self._reg, self._true, out=self._corr)

  def solve(self, rhs: np.ndarray, warm_start: np.ndarray) -> tuple[np.ndarray, dict[str, Any]]:
    np.copyto(self._rhs, rhs)
    self._rhs[self.n:] *= -1.0
    rhs_norm = np.linalg.norm(self._rhs, np.inf)
    tol = self._atol + self._rtol * rhs_norm
    sol = warm_start.copy()
    res = self._rhs - self._solver @ sol + self._corr * sol
    res_norm = np.linalg.norm(res, np.inf)
    status, solves = "non-converged", 0
    for solves in range(1, self.max_iterative_refinement_steps + 1):
      prev = res_norm
      sol += self._solver.solve(res)
      res = self._rhs - self._solver @ sol + self._corr * sol
      res_norm = np.linalg.norm(res, np.inf)
      if res_norm < tol:
        status = "converged"
        break
      if res_norm >= prev:
        logging.debug("IR stalled at step %d (%e -> %e)", solves, prev, res_norm)
        status = "stalled"
        break
    if np.any(np.isnan(sol)):
      raise ValueError("Linear solver returned NaNs.")
    return sol, {"solves": solves, "final_residual_norm": res_norm, "rhs_norm": rhs_norm,
                 "tolerance": tol, "converged": status == "converged", "status": status}

  def free(self) -> None:
    self._solver.free()
