"""Hot-path pieces on the device against the reference's own known answers
(tests/golden/reference_units.npz and reference_plugin.npz):

* Ruiz equilibration (qtqp_dense_equilibrate, the device IPM's first phase)
  against QTQP._equilibrate (src/qtqp/__init__.py:616-663) at the reference's
  own 1e-14 (tests/test_qtqp.py:1281-1296): d, e and the equilibrated A, P;
* the CudaDenseSolver plugin driven by the reference's refinement loop
  (tests/kkt_driver.py restates DirectKktSolver, src/qtqp/direct.py:112-311)
  against the reference's DirectKktSolver with its dense backend on the same
  seeded KKT systems: the same refinement outcome and solution.
"""

import numpy as np
import pytest

from qtqp_b200 import _lib, direct
from tests import golden_io, kkt_driver

pytestmark = pytest.mark.gpu

RUIZ_TOL = 1e-14  # tests/test_qtqp.py:1293-1296


@pytest.mark.parametrize("k", range(3))
def test_device_ruiz_matches_reference(k):
  import torch
  lib = _lib.load()
  g = golden_io.load("reference_units.npz")
  pre = f"ruiz{k}/"
  # Row-major copies (a CSC matrix's toarray() is column-major).
  a = np.ascontiguousarray(golden_io.csc(g, pre + "a").toarray())
  p = np.ascontiguousarray(golden_io.csc(g, pre + "p").toarray())
  m, n = a.shape
  dev = dict(dtype=torch.float64, device="cuda")
  da, dp = torch.from_numpy(a).to(**dev), torch.from_numpy(p).to(**dev)
  db, dc = torch.from_numpy(g[pre + "b"]).to(**dev), torch.from_numpy(g[pre + "c"]).to(**dev)
  ws = torch.empty(lib.qtqp_kkt_dense_workspace_bytes(n, m), dtype=torch.uint8, device="cuda")
  d_out, e_out = torch.empty(m, **dev), torch.empty(n, **dev)
  a_eq, p_eq = torch.empty(m * n, **dev), torch.empty(n * n, **dev)
  _lib.check(lib.qtqp_dense_equilibrate(
      n, m, da.data_ptr(), dp.data_ptr(), db.data_ptr(), dc.data_ptr(), ws.data_ptr(),
      d_out.data_ptr(), e_out.data_ptr(), a_eq.data_ptr(), p_eq.data_ptr(),
      _lib.stream_handle(torch.cuda.current_stream())))
  torch.cuda.synchronize()
  tol = dict(rtol=RUIZ_TOL, atol=RUIZ_TOL)
  np.testing.assert_allclose(d_out.cpu().numpy(), g[pre + "d"], **tol)
  np.testing.assert_allclose(e_out.cpu().numpy(), g[pre + "e"], **tol)
  np.testing.assert_allclose(a_eq.cpu().numpy().reshape(m, n), g[pre + "a_eq"], **tol)
  np.testing.assert_allclose(p_eq.cpu().numpy().reshape(n, n), g[pre + "p_eq"], **tol)


@pytest.mark.parametrize("k", range(4))
def test_plugin_in_refinement_driver_matches_reference(k):
  g = golden_io.load("reference_plugin.npz")
  pre = f"plugin{k}/"
  a, p = golden_io.csc(g, pre + "a"), golden_io.csc(g, pre + "p")
  m, n = a.shape
  z, mu = int(g[pre + "z"]), float(g[pre + "mu"])
  kkt = kkt_driver.DirectKktSolver(a=a, p=p, z=z, min_static_regularization=1e-8,
                                   max_iterative_refinement_steps=20, atol=1e-12, rtol=1e-12,
                                   solver=direct.CudaDenseSolver())
  try:
    kkt.update(mu=mu, s=g[pre + "s"], y=g[pre + "y"])
    sol, st = kkt.solve(rhs=g[pre + "rhs"], warm_start=np.zeros(n + m))
  finally:
    kkt.free()
  ref = g[pre + "dense/sol"]
  assert st["status"] == str(g[pre + "dense/status"])
  assert abs(st["solves"] - int(g[pre + "dense/solves"])) <= 1
  assert st["final_residual_norm"] < st["tolerance"]
  # Both sides refine to a 1e-12 residual, so they agree to the system's
  # conditioning; the reference's two backends agree to the same bound.
  scale = np.abs(ref).max()
  other = g[pre + "superlu/sol"]
  bound = max(10 * np.abs(ref - other).max(), 1e-10 * scale)
  np.testing.assert_allclose(sol, ref, rtol=0, atol=bound)
