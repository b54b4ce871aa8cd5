"""One sparse QP on the whole GPU with a supernodal Cholesky of its Gram matrix.

For QPs whose Gram matrix P + A^T D A is neither small and dense nor
narrow-banded: the role of the reference's sparse direct backends
(src/qtqp/solvers_sparse.py:96-121, src/qtqp/solvers_gpu.py:27-116).  The
host symbolic stage (libqtqp_cuda ``qtqp_sparse_analyze``: minimum-degree
ordering, elimination tree, supernodes, update lists, the grid's schedule)
runs once per sparsity pattern; the device IPM (``qtqp_sparse_grid_solve``)
assembles, factorises and solves with the supernodes on the whole GPU every
iteration.  The QP travels in the banded backend's pools (A as CSR and CSC, P
as CSR) with its variables in the plan's order; x comes back in that order and
is permuted to the caller's.
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp

from . import _lib
from . import band as _band
from .batch import SolveOptions


class SparsePlan:
  """Symbolic plan of one sparsity pattern of (A, P): the column order
  (perm[new] = old), the supernodes and the grid's schedule, packed in two
  pools for the device.  ordering: 'amd' (minimum degree) or 'natural'."""

  def __init__(self, a: sp.spmatrix, p: sp.spmatrix | None, ordering: str = "amd"):
    if ordering not in ("amd", "natural"):
      raise ValueError("ordering must be 'amd' or 'natural'")
    lib = _lib.load()
    a = sp.csc_matrix(a)
    m, n = a.shape
    a_ptr = np.ascontiguousarray(a.indptr, dtype=np.int32)
    a_idx = np.ascontiguousarray(a.indices, dtype=np.int32)
    p_ptr = p_idx = None
    if p is not None and p.nnz:
      pc = sp.csc_matrix(p)
      p_ptr = np.ascontiguousarray(pc.indptr, dtype=np.int32)
      p_idx = np.ascontiguousarray(pc.indices, dtype=np.int32)
    blocks = int(lib.qtqp_sparse_grid_blocks())
    desc = _lib.SparseDesc()
    handle = ctypes.c_void_p()
    _lib.check(lib.qtqp_sparse_analyze(
        n, m, a_ptr.ctypes.data, a_idx.ctypes.data if a_idx.size else None,
        p_ptr.ctypes.data if p_ptr is not None else None,
        p_idx.ctypes.data if p_idx is not None and p_idx.size else None,
        1 if ordering == "amd" else 0, blocks, ctypes.byref(handle), ctypes.byref(desc)))
    try:
      self.perm = np.empty(n, dtype=np.int32)
      self.pool32 = np.empty(max(int(desc.n32), 4), dtype=np.int32)
      self.pool64 = np.empty(max(int(desc.n64), 2), dtype=np.int64)
      _lib.check(lib.qtqp_sparse_export(handle, ctypes.byref(desc), self.perm.ctypes.data,
                                        self.pool32.ctypes.data, self.pool64.ctypes.data))
    finally:
      lib.qtqp_sparse_free(handle)
    self.desc = desc
    self.n, self.m = n, m

  @property
  def nnz_l(self) -> int:
    """Stored lower entries of the factor (explicit zeros of amalgamation included)."""
    return int(self.desc.nnz_l)

  @property
  def flops(self) -> float:
    """Floating-point operations of one numeric factorisation."""
    return float(self.desc.flops)

  def fill_fraction(self) -> float:
    """nnz(L) / the n (n + 1) / 2 entries of a dense factor."""
    return self.nnz_l / (0.5 * self.n * (self.n + 1))

  def section(self, name: str) -> np.ndarray:
    """One array of the plan by its descriptor name (host copy, for tests)."""
    d = self.desc
    sizes = {"first": d.nsuper + 1, "colsn": d.n, "rows": d.nrows, "upd_ptr": d.nsuper + 1,
             "upd_src": d.nupd, "upd_off": d.nupd, "upd_cnt": d.nupd,
             "cta_ptr": d.blocks + 1, "cta_range": 2 * d.nranges,
             "top_ptr": d.top_levels + 1, "top_list": d.ntop, "top_slab": d.ntop + 1,
             "gcol": d.ngram,
             "grow": d.ngram, "rowptr": d.nsuper + 1, "valptr": d.nsuper + 1,
             "gpos": d.ngram}
    off = int(getattr(d, "o_" + name))
    pool = self.pool64 if name in ("rowptr", "valptr", "gpos") else self.pool32
    return pool[off:off + int(sizes[name])]

  def permuted(self, a: sp.spmatrix, b, c, z: int, p: sp.spmatrix | None) -> _band.BandProblem:
    """The QP with its variables in the plan's order (the device's input)."""
    perm = self.perm
    a_p = sp.csc_matrix(sp.csc_matrix(a)[:, perm])
    p_p = sp.csc_matrix(sp.csc_matrix(p)[perm][:, perm]) if p is not None and p.nnz else None
    return _band.BandProblem(a_p, b, np.asarray(c, dtype=np.float64)[perm], z, p_p)

  def unpermute(self, x_plan: np.ndarray) -> np.ndarray:
    x = np.empty_like(x_plan)
    x[self.perm] = x_plan
    return x


class DeviceSparseGrid:
  """One sparse QP solved by the whole GPU (cooperative grid launch with the
  supernodal factorisation).  prob: the QP in the plan's column order
  (SparsePlan.permuted); same outputs as the banded grid solve, x in the
  plan's order."""

  def __init__(self, prob: _band.BandProblem, plan: SparsePlan, opts: SolveOptions,
               device=None, records: bool | None = None):
    torch = _lib.require_device()
    self.torch, self.plan, self.opts = torch, plan, opts
    dev = torch.device(device or "cuda")
    self.device = dev
    lib = _lib.load()
    pools = _band.BandPools([prob], opts)
    self.pools = pools
    self._inst = np.ascontiguousarray(pools.inst[:1])
    self.ws_bytes = int(lib.qtqp_sparse_grid_workspace_bytes(self._inst.ctypes.data,
                                                             ctypes.byref(plan.desc)))
    if self.ws_bytes == 0:
      msg = lib.qtqp_last_error()
      raise ValueError(msg.decode() if msg else "qtqp_sparse_grid_workspace_bytes failed")
    f64 = dict(dtype=torch.float64, device=dev)
    self.h_pools = [torch.from_numpy(x).pin_memory() for x in
                    (pools.ipool, pools.vpool, pools.b_pool, pools.c_pool)]
    self.ipool = torch.empty(pools.ipool.size, dtype=torch.int32, device=dev)
    self.vpool = torch.empty(pools.vpool.size, **f64)
    self.b = torch.empty(pools.b_pool.size, **f64)
    self.c = torch.empty(pools.c_pool.size, **f64)
    self.sn32 = torch.from_numpy(plan.pool32).to(dev)
    self.sn64 = torch.from_numpy(plan.pool64).to(dev)
    self.x = torch.empty(max(pools.n_total, 1), **f64)
    self.y = torch.empty(max(pools.m_total, 1), **f64)
    self.s = torch.empty(max(pools.m_total, 1), **f64)
    self.result = torch.zeros(_lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    self.stats = None
    if records or (records is None and opts.collect_stats):
      self.stats = torch.empty(opts.max_iter * _lib.STATS_DOUBLES, **f64)
    self._ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=dev)
    self.ws_ptr = (self._ws.data_ptr() + 255) & ~255
    self._copts = opts.to_c()

  @property
  def input_bytes(self) -> int:
    return sum(int(x.nbytes) for x in (self.pools.ipool, self.pools.vpool, self.pools.b_pool,
                                       self.pools.c_pool))

  def upload(self, stream=None) -> None:
    torch = self.torch
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip((self.ipool, self.vpool, self.b, self.c), self.h_pools):
        dst.copy_(src, non_blocking=True)

  def launch(self, stream=None) -> None:
    torch = self.torch
    st = stream or torch.cuda.current_stream(self.device)
    lib = _lib.load()
    _lib.check(lib.qtqp_sparse_grid_solve(
        self._inst.ctypes.data, ctypes.byref(self.plan.desc), self.sn32.data_ptr(),
        self.sn64.data_ptr(), self.ipool.data_ptr(), self.vpool.data_ptr(), self.b.data_ptr(),
        self.c.data_ptr(), self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(),
        self.result.data_ptr(), self.stats.data_ptr() if self.stats is not None else None,
        self.ws_ptr, self.ws_bytes, ctypes.byref(self._copts), _lib.stream_handle(st)))

  def fetch(self):
    """(results[1], x (plan order), y, s, stats or None) on the host."""
    self.torch.cuda.synchronize(self.device)
    res = self.result.cpu().numpy().view(_lib.RESULT_DTYPE)[:1]
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(1, self.opts.max_iter, _lib.STATS_DOUBLES)
    return res, self.x.cpu().numpy(), self.y.cpu().numpy(), self.s.cpu().numpy(), stats
