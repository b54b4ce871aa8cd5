"""KKT plugin interface and the CUDA dense backend.

``LinearSolver`` is the backend contract of the reference
(src/qtqp/direct.py:49-109): set_dims / set_kkt / update_diag / factorize /
solve / __matmul__ / format / free.  ``CudaDenseSolver`` implements it on the
GPU through the C-ABI (Gram/Schur reduction + Cholesky, the algorithm of
src/qtqp/solvers_dense.py:25-145), so it can be plugged into the reference's
own ``DirectKktSolver`` (direct.py:112-311), which drives the FP64 iterative
refinement around it.

The reference's other backends (SuperLU, PARDISO, CHOLMOD, cuDSS, ... in
src/qtqp/solvers_*.py) wrap CPU or vendor libraries that this build does not
ship; their enum names exist for drop-in use and raise ImportError when
instantiated, which is what the reference raises for a backend whose library
is not installed.
"""

from __future__ import annotations

import ctypes
from typing import Literal

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


def _unavailable(name: str, ref: str) -> type:
  """A backend class of the reference that this build does not ship."""

  def __init__(self, *args, **kwargs):
    raise ImportError(f"{name} ({ref}) is not part of the B200 build: use "
                      "LinearSolver.CUDA (or AUTO)")

  return type(name, (LinearSolver,), {"__init__": __init__, "__doc__": f"Not shipped: {ref}."})


AccelerateSolver = _unavailable("AccelerateSolver", "solvers_sparse.py, Apple Accelerate")
ScipySolver = _unavailable("ScipySolver", "solvers_sparse.py, SciPy SuperLU")
ScipyDenseSolver = _unavailable("ScipyDenseSolver", "solvers_dense.py, LAPACK potrf")
CupyDenseSolver = _unavailable("CupyDenseSolver", "solvers_gpu.py, CuPy")
UmfpackSolver = _unavailable("UmfpackSolver", "solvers_sparse.py, UMFPACK")
MklPardisoSolver = _unavailable("MklPardisoSolver", "solvers_sparse.py, MKL PARDISO")
QdldlSolver = _unavailable("QdldlSolver", "solvers_sparse.py, QDLDL")
CholModSolver = _unavailable("CholModSolver", "solvers_sparse.py, CHOLMOD")
CuDssSolver = _unavailable("CuDssSolver", "solvers_gpu.py, cuDSS")
EigenSolver = _unavailable("EigenSolver", "solvers_sparse.py, Eigen")
MumpsSolver = _unavailable("MumpsSolver", "solvers_sparse.py, MUMPS")
