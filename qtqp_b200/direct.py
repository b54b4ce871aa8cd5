"""KKT plugin interface and the CUDA dense backend.

``LinearSolver`` is the backend contract of the reference
(src/qtqp/direct.py:49-109): set_dims / set_kkt / update_diag / factorize /
solve / __matmul__ / format / free.  ``CudaDenseSolver`` implements it on the
GPU through the C-ABI (Gram/Schur reduction + Cholesky, the algorithm of
src/qtqp/solvers_dense.py:25-145), so it can be plugged into the reference's
own ``DirectKktSolver``.  ``DirectKktSolver`` here is the host-side refinement
driver with the reference's semantics (direct.py:112-311), used to exercise a
plugin in isolation.
"""

from __future__ import annotations

import ctypes
import logging
from typing import Any, Literal

import numpy as np
import scipy.sparse as sp

from . import _lib


def diag_data_indices(mat: sp.spmatrix) -> np.ndarray:
  """Data-array position of each diagonal entry of a CSC/CSR matrix
  (direct.py:33-46); vectorised over the columns."""
  mat.sort_indices()
  dim = mat.shape[0]
  ptr = mat.indptr
  counts = np.diff(ptr)
  owner = np.repeat(np.arange(dim), counts)
  hit = np.nonzero(mat.indices == owner)[0]
  out = np.empty(dim, dtype=np.intp)
  out[owner[hit]] = hit
  return out


class LinearSolver:
  """Backend contract for the quasi-definite KKT system (direct.py:49-109)."""

  def set_dims(self, n: int, m: int, z: int) -> None:
    pass

  def set_kkt(self, kkt: sp.spmatrix) -> None:
    self._kkt = kkt
    self._kkt_diag = kkt.diagonal()
    self._kkt_diag_idxs = diag_data_indices(kkt)

  def update_diag(self, diag: np.ndarray) -> None:
    self._kkt.data[self._kkt_diag_idxs] = diag
    np.copyto(self._kkt_diag, diag)

  def factorize(self) -> None:
    raise NotImplementedError

  def solve(self, rhs: np.ndarray) -> np.ndarray:
    raise NotImplementedError

  def __matmul__(self, x: np.ndarray) -> np.ndarray:
    res = self._kkt @ x
    res += self._kkt.T @ x
    res -= self._kkt_diag * x
    return res

  def format(self) -> str:
    raise NotImplementedError

  def free(self) -> None:
    pass


class CudaDenseSolver(LinearSolver):
  """Dense Gram/Cholesky KKT backend on the GPU (hand-written sm_100a kernels).

  Drop-in for the reference plugin API: host numpy vectors in and out, device
  buffers owned by the backend.  ``precision='mixed'`` factorises G in FP32;
  the caller's FP64 refinement (DirectKktSolver) recovers the accuracy.
  Raises ImportError/OSError when the library or a GPU is missing (the
  reference's AUTO resolution catches exactly these, __init__.py:72).
  """

  def __init__(self, precision: str = "fp64"):
    self._torch = _lib.require_device()
    self._lib = _lib.load()
    if precision not in ("fp64", "mixed"):
      raise ValueError("precision must be 'fp64' or 'mixed'")
    self._prec = _lib.PREC_FP64 if precision == "fp64" else _lib.PREC_MIXED
    self._ws = None
    self._n = self._m = 0

  def set_dims(self, n: int, m: int, z: int) -> None:
    torch = self._torch
    self._n, self._m = n, m
    nbytes = self._lib.qtqp_kkt_dense_workspace_bytes(n, m)
    if nbytes == 0:
      raise ValueError("CudaDenseSolver needs n >= 1 and m >= 1")
    dev = torch.device("cuda")
    self._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    self._diag = torch.empty(n + m, dtype=torch.float64, device=dev)
    self._vin = torch.empty(n + m, dtype=torch.float64, device=dev)
    self._vout = torch.empty(n + m, dtype=torch.float64, device=dev)
    self._info = torch.zeros(1, dtype=torch.int32, device=dev)
    self._host_out = torch.empty(n + m, dtype=torch.float64).pin_memory()

  def _stream(self) -> int:
    return _lib.stream_handle(self._torch.cuda.current_stream())

  def set_kkt(self, kkt: sp.spmatrix) -> None:
    super().set_kkt(kkt)
    n = self._n
    up = kkt.tocsr()
    a = np.ascontiguousarray(up[:n, n:].toarray().T, dtype=np.float64)
    p_up = up[:n, :n].toarray()
    p_full = p_up + p_up.T - np.diag(np.diag(p_up))
    np.fill_diagonal(p_full, 0.0)
    torch = self._torch
    self._a_dev = torch.from_numpy(a).cuda()
    self._p_dev = torch.from_numpy(np.ascontiguousarray(p_full)).cuda()
    _lib.check(self._lib.qtqp_kkt_dense_set(n, self._m, self._a_dev.data_ptr(),
                                            self._p_dev.data_ptr(), self._ws.data_ptr(),
                                            self._stream()))

  def update_diag(self, diag: np.ndarray) -> None:
    self._diag.copy_(self._torch.from_numpy(np.ascontiguousarray(diag, np.float64)))

  def factorize(self) -> None:
    _lib.check(self._lib.qtqp_kkt_dense_factorize(
        self._n, self._m, self._diag.data_ptr(), self._prec, self._ws.data_ptr(),
        self._info.data_ptr(), self._stream()))
    info = int(self._info.item())
    if info != 0:
      raise np.linalg.LinAlgError(f"Cholesky failed (pivot {info} not positive)")

  def _apply(self, fn, v: np.ndarray) -> np.ndarray:
    self._vin.copy_(self._torch.from_numpy(np.ascontiguousarray(v, np.float64)))
    _lib.check(fn(self._n, self._m, self._vin.data_ptr(), self._vout.data_ptr(),
                  self._ws.data_ptr(), self._stream()))
    self._host_out.copy_(self._vout)
    return self._host_out.numpy().copy()

  def solve(self, rhs: np.ndarray) -> np.ndarray:
    return self._apply(self._lib.qtqp_kkt_dense_solve, rhs)

  def __matmul__(self, x: np.ndarray) -> np.ndarray:
    return self._apply(self._lib.qtqp_kkt_dense_matvec, x)

  def format(self) -> Literal["csr"]:
    return "csr"

  def free(self) -> None:
    self._ws = None
    self._a_dev = self._p_dev = None


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
