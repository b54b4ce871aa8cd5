"""One large dense QP solved by the whole GPU through the C-ABI.

The device IPM runs in grid mode: one cooperative launch whose CTAs share the
interior-point loop (grid barriers and reductions), with the KKT Gram matrix
formed on the tensor cores (TF32 split into hi + lo, FP32 accumulation) for
the mixed-precision factor, or in FP64 for the plain factor, then a blocked
Cholesky and blocked triangular solves.  Same algorithm, options and outputs
as the batched paths (``qtqp_b200.batch``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import batch as _batch
from .batch import SolveOptions


class DeviceLarge:
  """Device buffers of one large dense QP and its workspace (torch tensors).

  prob is a QTQP (its CSC matrices are read column by column: a CSC matrix
  holding every entry is used in place, anything else is expanded column-major
  once) or a DenseProblem.  A and P travel to the device column-major and the
  solve reads them so; no host transpose."""

  def __init__(self, prob, opts: SolveOptions, device=None, records: bool | None = None):
    torch = _lib.require_device()
    self.torch, self.prob, self.opts = torch, prob, opts
    dev = torch.device(device or "cuda")
    self.device = dev
    pk = _batch._pack_of(prob)  # pylint: disable=protected-access
    n, m = pk.n, pk.m
    self.n, self.m, self.z = n, m, int(pk.z)
    self.has_p = pk.p_vals is not None
    self.flags = _lib.LARGE_COLMAJOR | (_lib.LARGE_HAS_P if self.has_p else 0)
    f64 = dict(dtype=torch.float64, device=dev)
    self.h_a = torch.from_numpy(pk.a_vals).pin_memory()
    self.h_p = torch.from_numpy(pk.p_vals).pin_memory() if self.has_p else None
    self.h_b = torch.from_numpy(np.ascontiguousarray(prob.b, dtype=np.float64)).pin_memory()
    self.h_c = torch.from_numpy(np.ascontiguousarray(prob.c, dtype=np.float64)).pin_memory()
    self.a = torch.empty(m * n, **f64)
    self.p = torch.empty(n * n, **f64) if self.has_p else None
    self.b = torch.empty(m, **f64)
    self.c = torch.empty(n, **f64)
    self.x = torch.empty(n, **f64)
    self.y = torch.empty(m, **f64)
    self.s = torch.empty(m, **f64)
    self.result = torch.zeros(_lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    self.stats = None
    if records or (records is None and opts.collect_stats):
      self.stats = torch.empty(opts.max_iter * _lib.STATS_DOUBLES, **f64)
    lib = _lib.load()
    self.ws_bytes = int(lib.qtqp_dense_large_workspace_bytes(n, m))
    # 1024-byte alignment for the tensor-core operands inside the workspace.
    self._ws = torch.empty(self.ws_bytes + 1024, dtype=torch.uint8, device=dev)
    self.ws_ptr = (self._ws.data_ptr() + 1023) & ~1023
    self._copts = opts.to_c()

  @property
  def input_bytes(self) -> int:
    return sum(int(t.numel() * t.element_size()) for t in
               (self.h_a, self.h_p, self.h_b, self.h_c) if t is not None)

  def upload(self, stream=None) -> None:
    torch = self.torch
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in ((self.a, self.h_a), (self.p, self.h_p), (self.b, self.h_b),
                       (self.c, self.h_c)):
        if src is not None:
          dst.copy_(src, non_blocking=True)

  def launch(self, stream=None) -> None:
    torch = self.torch
    st = stream or torch.cuda.current_stream(self.device)
    lib = _lib.load()
    _lib.check(lib.qtqp_dense_large_solve(
        self.n, self.m, self.z, self.flags, self.a.data_ptr(),
        self.p.data_ptr() if self.p is not None else None, self.b.data_ptr(),
        self.c.data_ptr(), self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(),
        self.result.data_ptr(), self.stats.data_ptr() if self.stats is not None else None,
        self.ws_ptr, self.ws_bytes, ctypes.byref(self._copts), _lib.stream_handle(st)))

  def fetch(self):
    """(results[1], x, y, s, stats or None) on the host, like the batches."""
    self.torch.cuda.synchronize(self.device)
    res = self.result.cpu().numpy().view(_lib.RESULT_DTYPE)[:1]
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(1, self.opts.max_iter, _lib.STATS_DOUBLES)
    return res, self.x.cpu().numpy(), self.y.cpu().numpy(), self.s.cpu().numpy(), stats
