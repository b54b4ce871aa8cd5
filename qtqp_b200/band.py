"""Batched banded/sparse device solve through the C-ABI.

For QPs whose Gram matrix ``P + A^T D A`` has a small half-bandwidth (such as
stage-ordered MPC problems), A is packed as CSR and CSC and P as CSR, and the
device IPM factorises the Gram matrix in band storage.  Same algorithm,
options and outputs as the dense batch (``qtqp_b200.batch``).
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import scipy.sparse as sp

from . import _lib
from .batch import SolveOptions


def gram_bandwidth(a: sp.spmatrix, p: sp.spmatrix | None) -> int:
  """Half-bandwidth of P + A^T D A for any positive diagonal D: the widest
  column span of a row of A, or of P's entries from the diagonal."""
  a = sp.csr_matrix(a)
  bw = 0
  if a.nnz:
    if not a.has_sorted_indices:
      a = a.sorted_indices()
    cnt = np.diff(a.indptr)
    rows = np.flatnonzero(cnt)
    lo = a.indices[a.indptr[rows]]
    hi = a.indices[a.indptr[rows + 1] - 1]
    bw = int(np.max(hi - lo))
  if p is not None and p.nnz:
    pc = sp.coo_matrix(p)
    bw = max(bw, int(np.max(np.abs(pc.row - pc.col))))
  return bw


def wide_by_counts(a: sp.spmatrix, p: sp.spmatrix | None, n: int) -> bool:
  """True when the Gram matrix has half-bandwidth above n/4 - 1 in every
  ordering of the variables, read from entry counts alone: a row of A with k
  entries spans at least k columns, and a column of P with k entries reaches
  at least (k - 1) / 2 from the diagonal."""
  if a.nnz:
    rows = np.bincount(a.indices, minlength=a.shape[0]) if a.format == "csc" else \
        np.diff(sp.csr_matrix(a).indptr)
    if 4 * int(rows.max()) > n:
      return True
  if p is not None and p.nnz:
    cols = np.diff(sp.csc_matrix(p).indptr)
    if 2 * (int(cols.max()) + 1) > n:
      return True
  return False


def band_ordering(a: sp.spmatrix, p: sp.spmatrix | None):
  """A reverse Cuthill-McKee ordering of the variables for the sparsity graph
  of P + A^T A (variables adjacent when they share a row of A or an entry of
  P), or None when A is dense or that graph holds more than a quarter of
  the n x n entries (no narrow ordering to find)."""
  from scipy.sparse import csgraph  # pylint: disable=g-import-not-at-top
  m, n = a.shape
  if a.nnz > 0.1 * float(m) * n:  # dense A: a dense Gram, no narrow ordering
    return None
  ab = sp.csr_matrix(a, dtype=np.float64, copy=True)
  ab.data[:] = 1.0
  g = (ab.T @ ab).tocsr()
  if g.nnz > 0.25 * float(n) * n:
    return None
  if p is not None and p.nnz:
    pb = sp.csr_matrix(p, dtype=np.float64, copy=True)
    pb.data[:] = 1.0
    g = (g + pb).tocsr()
  g = g + sp.eye(n, format="csr")
  return np.asarray(csgraph.reverse_cuthill_mckee(g, symmetric_mode=True), dtype=np.int64)


class _Structure:
  """CSR / CSC / P arrays and bandwidth of one (A, P) pair."""

  def __init__(self, a: sp.spmatrix, p: sp.spmatrix | None):
    self.src = (a, p)  # keeps the sources alive while the cache refers to them
    self.a = sp.csr_matrix(a, dtype=np.float64)
    self.a.sort_indices()
    self.at = sp.csr_matrix(self.a.T)  # CSC of A = CSR of A^T
    self.at.sort_indices()
    self.p = None
    if p is not None and sp.csr_matrix(p).nnz:
      self.p = sp.csr_matrix(p, dtype=np.float64)
      self.p.sort_indices()
    self.bw = gram_bandwidth(self.a, self.p)


_STRUCT_CACHE: dict = {}


def _structure(a, p) -> _Structure:
  """Converted structure of (a, p), shared by every problem built from the
  same matrix objects (a parametric family converts A and P once)."""
  key = (id(a), id(p))
  hit = _STRUCT_CACHE.get(key)
  if hit is not None and hit.src[0] is a and hit.src[1] is p:
    return hit
  if len(_STRUCT_CACHE) > 64:
    _STRUCT_CACHE.clear()
  st = _Structure(a, p)
  _STRUCT_CACHE[key] = st
  return st


class BandProblem:
  """One presolved sparse QP (A, P as scipy matrices; P may be None).
  Problems built from the same A and P objects share one packed copy."""

  def __init__(self, a: sp.spmatrix, b, c, z: int, p: sp.spmatrix | None = None):
    self.structure = _structure(a, p)
    self.a, self.at, self.p = self.structure.a, self.structure.at, self.structure.p
    self.b = np.asarray(b, dtype=np.float64)
    self.c = np.asarray(c, dtype=np.float64)
    self.z = int(z)
    self.bw = self.structure.bw


class BandPools:
  """Descriptors and packed int32 / double pools of sparse QPs (A as CSR and
  CSC, P as CSR), the input layout of the banded and supernodal solves."""

  def __init__(self, problems: Sequence[BandProblem], opts: SolveOptions):
    count = len(problems)
    self.count = count
    inst = np.zeros(count, dtype=_lib.BAND_DTYPE)
    ints, vals = [], []
    ioff = voff = n_off = m_off = 0

    def put_i(arr):
      nonlocal ioff
      ints.append(np.asarray(arr, dtype=np.int32))
      o = ioff
      ioff += len(arr)
      return o

    def put_v(arr):
      nonlocal voff
      vals.append(np.asarray(arr, dtype=np.float64))
      o = voff
      voff += len(arr)
      return o

    packed = {}  # id(structure) -> offsets of its shared A / P arrays
    for i, pr in enumerate(problems):
      m, n = pr.a.shape
      d = inst[i]
      d["n"], d["m"], d["z"] = n, m, pr.z
      d["has_p"] = int(pr.p is not None)
      d["bw"] = min(pr.bw, n - 1)
      d["nnz_a"] = pr.a.nnz
      d["nnz_p"] = pr.p.nnz if pr.p is not None else 0
      key = id(pr.structure)
      if key not in packed:
        offs = {"a_ptr": put_i(pr.a.indptr), "a_idx": put_i(pr.a.indices),
                "a_val": put_v(pr.a.data), "at_ptr": put_i(pr.at.indptr),
                "at_idx": put_i(pr.at.indices), "at_val": put_v(pr.at.data)}
        if pr.p is not None:
          offs.update(p_ptr=put_i(pr.p.indptr), p_idx=put_i(pr.p.indices),
                      p_val=put_v(pr.p.data))
        else:
          offs.update(p_ptr=put_i(np.zeros(n + 1, dtype=np.int32)), p_idx=0, p_val=0)
        packed[key] = offs
      for name, off in packed[key].items():
        d[name] = off
      d["n_off"], d["m_off"] = n_off, m_off
      d["st_off"] = i * opts.max_iter
      n_off += n
      m_off += m
    self.ipool = np.concatenate(ints) if ints else np.zeros(1, np.int32)
    self.vpool = np.concatenate(vals) if vals else np.zeros(1)
    self.b_pool = np.concatenate([pr.b for pr in problems]) if count else np.zeros(1)
    self.c_pool = np.concatenate([pr.c for pr in problems]) if count else np.zeros(1)
    self.n_total, self.m_total = n_off, m_off
    self.inst, self.opts = inst, opts


class HostBandBatch(BandPools):
  """Packed int32/double pools, descriptors and plan of a banded batch."""

  def __init__(self, problems: Sequence[BandProblem], opts: SolveOptions, num_sms: int = 0):
    super().__init__(problems, opts)
    lib = _lib.load()
    count = self.count
    order = np.zeros(max(count, 1), dtype=np.int32)
    plan = _lib.BatchPlan()
    copts = opts.to_c()
    _lib.check(lib.qtqp_band_batch_plan(self.inst.ctypes.data, count, ctypes.byref(copts),
                                        num_sms, order.ctypes.data, ctypes.byref(plan)))
    self.order, self.plan = order, plan
    self.workspace_bytes = int(plan.workspace_bytes)

  @property
  def input_bytes(self) -> int:
    return sum(int(x.nbytes) for x in (self.ipool, self.vpool, self.b_pool, self.c_pool))


class DeviceBandBatch:
  """Device copy of a HostBandBatch, outputs and workspace (torch tensors)."""

  def __init__(self, hb: HostBandBatch, device=None, records: bool | None = None):
    torch = _lib.require_device()
    self.torch, self.hb = torch, hb
    dev = torch.device(device or "cuda")
    self.device = dev
    f64 = dict(dtype=torch.float64, device=dev)
    self.inst = torch.from_numpy(hb.inst.view(np.uint8)).to(dev)
    self.order = torch.from_numpy(hb.order).to(dev)
    self.h_pools = [torch.from_numpy(x).pin_memory() for x in
                    (hb.ipool, hb.vpool, hb.b_pool, hb.c_pool)]
    self.ipool = torch.empty(hb.ipool.size, dtype=torch.int32, device=dev)
    self.vpool = torch.empty(hb.vpool.size, **f64)
    self.b = torch.empty(hb.b_pool.size, **f64)
    self.c = torch.empty(hb.c_pool.size, **f64)
    self.x = torch.empty(max(hb.n_total, 1), **f64)
    self.y = torch.empty(max(hb.m_total, 1), **f64)
    self.s = torch.empty(max(hb.m_total, 1), **f64)
    self.results = torch.empty(max(hb.count, 1) * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                               device=dev)
    self.stats = None
    if records or (records is None and hb.opts.collect_stats):
      self.stats = torch.empty(max(hb.count, 1) * hb.opts.max_iter * _lib.STATS_DOUBLES, **f64)
    self.workspace = torch.empty(hb.workspace_bytes, dtype=torch.uint8, device=dev)
    self._copts = hb.opts.to_c()

  def upload(self, stream=None) -> None:
    torch = self.torch
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip((self.ipool, self.vpool, self.b, self.c), self.h_pools):
        dst.copy_(src, non_blocking=True)

  def launch(self, stream=None, warm=None) -> None:
    """Enqueues the batch solve.  warm = (x, y, active) device tensors laid
    out like the x / y pools (FP64, FP64, uint8) enables the learned warm
    start; None runs the plain method."""
    torch = self.torch
    lib = _lib.load()
    st = stream or torch.cuda.current_stream(self.device)
    hb = self.hb
    wx = wy = wa = None
    if warm is not None:
      for t, numel, dt in zip(warm, (hb.n_total, hb.m_total, hb.m_total),
                              (torch.float64, torch.float64, torch.uint8)):
        if t.dtype != dt or t.numel() < numel or not t.is_contiguous() or not t.is_cuda:
          raise ValueError("warm start tensors must be contiguous (x f64, y f64, active u8) "
                           "on the batch's device, sized like the x / y pools")
      wx, wy, wa = (t.data_ptr() for t in warm)
    _lib.check(lib.qtqp_band_batch_solve(
        self.inst.data_ptr(), self.order.data_ptr(), ctypes.byref(hb.plan),
        self.ipool.data_ptr(), self.vpool.data_ptr(), self.b.data_ptr(), self.c.data_ptr(),
        self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(), self.results.data_ptr(),
        self.stats.data_ptr() if self.stats is not None else None,
        self.workspace.data_ptr(), hb.workspace_bytes, ctypes.byref(self._copts), wx, wy, wa,
        _lib.stream_handle(st)))

  def fetch(self):
    self.torch.cuda.synchronize(self.device)
    res = self.results.cpu().numpy().view(_lib.RESULT_DTYPE)[: self.hb.count]
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(self.hb.count, self.hb.opts.max_iter,
                                                _lib.STATS_DOUBLES)
    return (res, self.x.cpu().numpy(), self.y.cpu().numpy(), self.s.cpu().numpy(), stats)


# Widest band of the whole-GPU path (two bw x bw FP64 separator blocks
# staged in 225 KiB of shared memory).
GRID_MAX_BW = 118


def grid_supported(bw: int, n: int) -> bool:
  """Whether one banded QP of half-bandwidth bw can use the whole-GPU
  partitioned solve (the separator blocks must fit in shared memory)."""
  return 1 <= bw <= GRID_MAX_BW and n >= 2 * bw + 2


class DeviceBandGrid:
  """One banded QP solved by the whole GPU (cooperative grid launch with the
  partitioned band factorisation).  Takes a single-problem HostBandBatch for
  the packed pools and descriptor; same outputs as DeviceBandBatch."""

  def __init__(self, hb: HostBandBatch, device=None, records: bool | None = None,
               parts: int | None = None):
    if hb.count != 1:
      raise ValueError("DeviceBandGrid solves exactly one problem")
    torch = _lib.require_device()
    self.torch, self.hb = torch, hb
    dev = torch.device(device or "cuda")
    self.device = dev
    lib = _lib.load()
    self._inst = np.ascontiguousarray(hb.inst[:1])
    self.parts = int(lib.qtqp_band_grid_default_parts(self._inst.ctypes.data)
                     if parts is None else parts)
    self.ws_bytes = int(lib.qtqp_band_grid_workspace_bytes(self._inst.ctypes.data, self.parts))
    if self.ws_bytes == 0:
      msg = lib.qtqp_last_error()
      raise ValueError(msg.decode() if msg else "qtqp_band_grid_workspace_bytes failed")
    f64 = dict(dtype=torch.float64, device=dev)
    self.h_pools = [torch.from_numpy(x).pin_memory() for x in
                    (hb.ipool, hb.vpool, hb.b_pool, hb.c_pool)]
    self.ipool = torch.empty(hb.ipool.size, dtype=torch.int32, device=dev)
    self.vpool = torch.empty(hb.vpool.size, **f64)
    self.b = torch.empty(hb.b_pool.size, **f64)
    self.c = torch.empty(hb.c_pool.size, **f64)
    self.x = torch.empty(max(hb.n_total, 1), **f64)
    self.y = torch.empty(max(hb.m_total, 1), **f64)
    self.s = torch.empty(max(hb.m_total, 1), **f64)
    self.result = torch.zeros(_lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    self.stats = None
    if records or (records is None and hb.opts.collect_stats):
      self.stats = torch.empty(hb.opts.max_iter * _lib.STATS_DOUBLES, **f64)
    self._ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=dev)
    self.ws_ptr = (self._ws.data_ptr() + 255) & ~255
    self._copts = hb.opts.to_c()

  @property
  def input_bytes(self) -> int:
    return self.hb.input_bytes

  def upload(self, stream=None) -> None:
    torch = self.torch
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip((self.ipool, self.vpool, self.b, self.c), self.h_pools):
        dst.copy_(src, non_blocking=True)

  def launch(self, stream=None) -> None:
    torch = self.torch
    st = stream or torch.cuda.current_stream(self.device)
    lib = _lib.load()
    _lib.check(lib.qtqp_band_grid_solve(
        self._inst.ctypes.data, self.parts, self.ipool.data_ptr(), self.vpool.data_ptr(),
        self.b.data_ptr(), self.c.data_ptr(), self.x.data_ptr(), self.y.data_ptr(),
        self.s.data_ptr(), self.result.data_ptr(),
        self.stats.data_ptr() if self.stats is not None else None, self.ws_ptr, self.ws_bytes,
        ctypes.byref(self._copts), _lib.stream_handle(st)))

  def fetch(self):
    """(results[1], x, y, s, stats or None) on the host, like the batches."""
    self.torch.cuda.synchronize(self.device)
    res = self.result.cpu().numpy().view(_lib.RESULT_DTYPE)[:1]
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(1, self.hb.opts.max_iter, _lib.STATS_DOUBLES)
    return res, self.x.cpu().numpy(), self.y.cpu().numpy(), self.s.cpu().numpy(), stats
