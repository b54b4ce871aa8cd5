"""Device-resident batched solve of dense QPs through the C-ABI.

A batch is packed once into flat pools (column-major A and P per instance --
the value order of a CSC matrix that stores every entry, so a dense QP given
in CSC form packs without conversion -- then b and c), planned by the library
(processing order, launch shape, workspace), copied to the device, and solved
by one persistent launch of
``qtqp_dense_batch_solve``: one thread block runs one QP's whole interior-point
method (the device counterpart of ``QTQP._solve_impl``,
src/qtqp/__init__.py:351-614 of the reference).
"""

from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Sequence

import numpy as np
import scipy.sparse as sp

from . import _lib


@dataclasses.dataclass(frozen=True)
class SolveOptions:
  """Keyword arguments of QTQP.solve (src/qtqp/__init__.py:309-326) plus the
  device-only precision switch."""

  atol: float = 1e-7
  rtol: float = 1e-8
  atol_infeas: float = 1e-8
  rtol_infeas: float = 1e-9
  max_iter: int = 100
  step_size_scale: float = 0.99
  min_static_regularization: float = 1e-8
  max_iterative_refinement_steps: int = 20
  linear_solver_atol: float = 1e-12
  linear_solver_rtol: float = 1e-12
  equilibrate: bool = True
  collect_stats: bool = False
  precision: str = "fp64"  # "fp64" or "mixed"
  tau_mode: int = 0
  warm_corrections: int = 0  # learned warm start: active-set corrections
  warm_shift: float = 0.0  # learned warm start: > 0 starts a rejected instance's IPM there

  def validate(self) -> None:
    """The reference's argument checks (__init__.py:403-412)."""
    assert self.atol >= 0
    assert self.rtol >= 0
    assert self.atol_infeas >= 0
    assert self.rtol_infeas >= 0
    assert self.max_iter > 0
    assert 0 < self.step_size_scale < 1
    assert self.min_static_regularization >= 0
    assert self.max_iterative_refinement_steps >= 1
    assert self.linear_solver_atol >= 0
    assert self.linear_solver_rtol >= 0
    assert 0 <= self.warm_corrections <= 64
    assert self.warm_shift >= 0
    if self.precision not in ("fp64", "mixed"):
      raise ValueError(f"precision must be 'fp64' or 'mixed', got {self.precision!r}")

  def to_c(self) -> _lib.Options:
    return _lib.Options(
        self.atol, self.rtol, self.atol_infeas, self.rtol_infeas,
        self.step_size_scale, self.min_static_regularization,
        self.linear_solver_atol, self.linear_solver_rtol, int(self.max_iter),
        int(self.max_iterative_refinement_steps), int(bool(self.equilibrate)),
        _lib.PREC_FP64 if self.precision == "fp64" else _lib.PREC_MIXED,
        int(bool(self.collect_stats)), int(self.tau_mode), int(self.warm_corrections),
        float(self.warm_shift))


@dataclasses.dataclass
class DenseProblem:
  """One presolved QP in dense form: A (m x n), P (n x n) or None, b, c, z."""

  a: np.ndarray
  b: np.ndarray
  c: np.ndarray
  z: int
  p: np.ndarray | None = None


class _Pack:
  """Column-major FP64 values of one QP's A and P (P: None when it is zero)
  and their host addresses, ready for the gather into the batch pools."""

  __slots__ = ("src_a", "src_p", "n", "m", "z", "a_vals", "p_vals", "a_ptr", "p_ptr", "b", "c",
               "b_ptr", "c_ptr")

  def __init__(self, src_a, src_p, n, m, z, a_vals, p_vals, b, c):
    self.src_a, self.src_p = src_a, src_p
    self.n, self.m, self.z = n, m, z
    self.a_vals = a_vals
    self.p_vals = p_vals
    self.a_ptr = a_vals.ctypes.data
    self.p_ptr = 0 if p_vals is None else p_vals.ctypes.data
    self.b, self.c = b, c  # FP64, contiguous: gathered like A and P
    self.b_ptr, self.c_ptr = b.ctypes.data, c.ctypes.data


def _colmajor_values(mat, rows: int, cols: int) -> tuple[np.ndarray, bool]:
  """(values, zero_copy): the column-major dense values of a sparse or dense
  matrix.  A CSC matrix that stores every entry in canonical order already
  holds them in its data array (zero copy); anything else is densified."""
  if sp.issparse(mat):
    if (mat.format == "csc" and mat.nnz == rows * cols and mat.dtype == np.float64 and
        mat.has_canonical_format and mat.data.flags.c_contiguous):
      return mat.data, True
    return np.asarray(mat.toarray(order="F"), dtype=np.float64).ravel(order="F"), False
  return np.asarray(mat, dtype=np.float64).ravel(order="F"), False


def _pack_of(pr) -> _Pack:
  """The pack of a QTQP (cached on it while its A and P objects stay the same
  and their values can be read in place) or of a DenseProblem."""
  if isinstance(pr, DenseProblem):
    m, n = pr.a.shape
    a_vals, _ = _colmajor_values(pr.a, m, n)
    has_p = pr.p is not None and bool(np.any(pr.p != 0))
    p_vals = _colmajor_values(pr.p, n, n)[0] if has_p else None
    return _Pack(None, None, n, m, pr.z, a_vals, p_vals, _f64(pr.b), _f64(pr.c))
  pk = getattr(pr, "_dense_pack", None)
  if (pk is not None and pk.src_a is pr.a and pk.src_p is pr.p and pk.b is pr.b and
      pk.c is pr.c):
    return pk
  n, m = pr.n, pr.m
  a_vals, a_view = _colmajor_values(pr.a, m, n)
  p_vals, p_view = None, True
  if pr.p.nnz and np.any(pr.p.data != 0):  # the device needs P when it is non-zero
    p_vals, p_view = _colmajor_values(pr.p, n, n)
  b, c = _f64(pr.b), _f64(pr.c)
  pk = _Pack(pr.a, pr.p, n, m, pr.z, a_vals, p_vals, b, c)
  if a_view and p_view and b is pr.b and c is pr.c:  # read in place: valid while they are
    pr._dense_pack = pk  # pylint: disable=protected-access
  return pk


def _f64(v) -> np.ndarray:
  """v itself when it is a contiguous FP64 vector, else such a copy."""
  if (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.ndim == 1 and
      v.flags.c_contiguous):
    return v
  return np.ascontiguousarray(v, dtype=np.float64).reshape(-1)


def _gather(lib, pool: np.ndarray, ptrs, nbytes, offs) -> None:
  ptrs = np.ascontiguousarray(ptrs, dtype=np.uint64)
  nbytes = np.ascontiguousarray(nbytes, dtype=np.int64)
  offs = np.ascontiguousarray(offs, dtype=np.int64)
  if ptrs.size:
    _lib.check(lib.qtqp_host_gather(int(ptrs.size), ptrs.ctypes.data, nbytes.ctypes.data,
                                    offs.ctypes.data, pool.ctypes.data, 0))


class PinnedArena:
  """Pinned host buffers kept across calls (grown, never shrunk), for a caller
  that builds one batch at a time: allocating and page-locking 150 MB of
  pools on every call costs more than the packing itself.  Whoever holds
  `lock` owns the buffers until it releases it."""

  def __init__(self):
    import threading  # pylint: disable=g-import-not-at-top
    self.lock = threading.Lock()
    self._bufs = {}

  def get(self, slot: str, count: int):
    import torch  # pylint: disable=g-import-not-at-top
    t = self._bufs.get(slot)
    if t is None or t.numel() < count:
      t = torch.empty(max(count, 1), dtype=torch.float64, pin_memory=True)
      self._bufs[slot] = t
    return t[:count]


class HostBatch:
  """Packed host pools of a batch: A and P column-major per instance, b, c.

  problems: QTQP objects (their CSC values are gathered in place when every
  entry is stored) or DenseProblems.  pinned=True allocates the pools in
  pinned host memory (torch), so that they are copied to the device
  asynchronously without a staging copy; pinned=<PinnedArena> takes them
  from the arena (the caller holds its lock while the batch lives).
  """

  def __init__(self, problems: Sequence, opts: SolveOptions, block_threads: int = 0,
               smem_bytes: int = 0, pinned: bool = False, tuning=None, defer: bool = False):
    count = len(problems)
    self.count = count
    packs = [_pack_of(pr) for pr in problems]
    ns = np.fromiter((pk.n for pk in packs), np.int64, count)
    ms = np.fromiter((pk.m for pk in packs), np.int64, count)
    has_p = np.fromiter((pk.p_ptr != 0 for pk in packs), np.bool_, count)
    inst = np.zeros(count, dtype=_lib.INSTANCE_DTYPE)
    inst["n"], inst["m"] = ns, ms
    inst["z"] = np.fromiter((pk.z for pk in packs), np.int64, count)
    inst["has_p"] = has_p
    inst["st_off"] = np.arange(count, dtype=np.int64) * opts.max_iter
    self.inst, self.opts = inst, opts
    self.order = np.zeros(max(count, 1), dtype=np.int32)
    self.replan(tuning, block_threads, smem_bytes)
    # Every pool is laid out in processing order, so that each launch group's
    # inputs and outputs are contiguous ranges (packed, copied and read back
    # per group by DeviceBatch.solve_pipelined / fetch_groups).
    pos = self.order[:count]
    a_sz, p_sz = ms * ns, np.where(has_p, ns * ns, 0)
    for key, sz in (("a_off", a_sz), ("p_off", p_sz), ("n_off", ns), ("m_off", ms)):
      srt = sz[pos]
      inst[key][pos] = np.cumsum(srt) - srt
    self._a_sz, self._p_sz, self._packs = a_sz, p_sz, packs
    a_total, p_total = int(a_sz.sum()), int(p_sz.sum())
    self.n_total, self.m_total = int(ns.sum()), int(ms.sum())
    self.pinned = pinned
    self.h_pools = None
    sizes = (max(a_total, 1), max(p_total, 1), max(self.m_total, 1), max(self.n_total, 1))
    self.arena = pinned if isinstance(pinned, PinnedArena) else None
    if isinstance(pinned, PinnedArena):
      self.h_pools = [pinned.get(slot, k) for slot, k in zip("apbc", sizes)]
      self.a_pool, self.p_pool, self.b_pool, self.c_pool = (t.numpy() for t in self.h_pools)
    elif pinned:
      import torch  # pylint: disable=g-import-not-at-top
      self.h_pools = [torch.empty(k, dtype=torch.float64, pin_memory=True) for k in sizes]
      self.a_pool, self.p_pool, self.b_pool, self.c_pool = (t.numpy() for t in self.h_pools)
    else:
      self.a_pool, self.p_pool, self.b_pool, self.c_pool = (np.empty(k) for k in sizes)
    if p_total == 0:
      self.p_pool[:] = 0.0
    self.gathered = False
    if not defer:
      self.gather_all()

  def gather_group(self, g: int):
    """Packs the A, P, b and c values of launch group g into the pools;
    returns the element ranges ((a_lo, a_hi), (p_lo, p_hi), (m_lo, m_hi),
    (n_lo, n_hi)) of its A, P, b and c."""
    lib = _lib.load()
    grp = self.plan.groups[g]
    ids = self.order[grp.begin:grp.begin + grp.count]
    if not len(ids):
      return (0, 0), (0, 0), (0, 0), (0, 0)
    inst, packs = self.inst, self._packs
    sel = [packs[i] for i in ids.tolist()]
    a_sz, p_sz = self._a_sz[ids], self._p_sz[ids]
    a_off, p_off = inst["a_off"][ids], inst["p_off"][ids]
    n_sz, m_sz = inst["n"][ids], inst["m"][ids]
    n_off, m_off = inst["n_off"][ids], inst["m_off"][ids]
    _gather(lib, self.a_pool, [pk.a_ptr for pk in sel], 8 * a_sz, 8 * a_off)
    has = np.nonzero(p_sz)[0]
    _gather(lib, self.p_pool, [sel[k].p_ptr for k in has.tolist()], 8 * p_sz[has],
            8 * p_off[has])
    _gather(lib, self.b_pool, [pk.b_ptr for pk in sel], 8 * m_sz, 8 * m_off)
    _gather(lib, self.c_pool, [pk.c_ptr for pk in sel], 8 * n_sz, 8 * n_off)
    a_rng = (int(a_off[0]), int(a_off[-1] + a_sz[-1]))
    p_rng = (int(p_off[0]), int(p_off[-1] + p_sz[-1]))
    m_rng = (int(m_off[0]), int(m_off[-1] + m_sz[-1]))
    n_rng = (int(n_off[0]), int(n_off[-1] + n_sz[-1]))
    return a_rng, p_rng, m_rng, n_rng

  def launch_order(self) -> list[int]:
    """Launch groups in increasing order of their packed A and P bytes."""
    sizes = []
    for g in range(self.plan.num_groups):
      grp = self.plan.groups[g]
      ids = self.order[grp.begin:grp.begin + grp.count]
      sizes.append((int(self._a_sz[ids].sum() + self._p_sz[ids].sum()), g))
    return [g for _, g in sorted(sizes)]

  def gather_all(self) -> None:
    """Packs every group's A and P values."""
    for g in range(self.plan.num_groups):
      self.gather_group(g)
    self.gathered = True

  def replan(self, tuning=None, block_threads: int = 0, smem_bytes: int = 0) -> None:
    """(Re)plans the launch groups: the library's default shapes, a forced
    shape (block_threads / smem_bytes), or a tuning table (a list of
    {n_lo, n_hi, block_threads, lean, onchip} entries, see autotune.py)."""
    lib = _lib.load()
    plan = _lib.BatchPlan()
    copts = self.opts.to_c()
    if tuning:
      table = (_lib.BatchTuning * len(tuning))(*[
          _lib.BatchTuning(int(e["n_lo"]), int(e["n_hi"]), int(e["block_threads"]),
                           int(e.get("lean", 0)), int(e.get("onchip", 0)), 0) for e in tuning])
      _lib.check(lib.qtqp_dense_batch_plan_tuned(self.inst.ctypes.data, self.count,
                                                 ctypes.byref(copts), self.order.ctypes.data,
                                                 table, len(tuning), ctypes.byref(plan)))
    else:
      _lib.check(lib.qtqp_dense_batch_plan(self.inst.ctypes.data, self.count,
                                           ctypes.byref(copts), self.order.ctypes.data,
                                           block_threads, smem_bytes, ctypes.byref(plan)))
    self.plan = plan
    self.workspace_bytes = int(plan.workspace_bytes)
    self.tuning = tuning

  @property
  def groups(self):
    """(begin, count, block_threads, smem_bytes) of each launch group."""
    return [(g.begin, g.count, g.block_threads, g.smem_bytes)
            for g in self.plan.groups[:self.plan.num_groups]]

  def group_n_range(self, g: int) -> tuple[int, int]:
    """Smallest and largest n of launch group g."""
    grp = self.plan.groups[g]
    ids = self.order[grp.begin:grp.begin + grp.count]
    ns = self.inst["n"][ids]
    return int(ns.min()), int(ns.max())

  @property
  def input_bytes(self) -> int:
    return sum(int(x.nbytes) for x in (self.a_pool, self.p_pool, self.b_pool, self.c_pool))


class DeviceBatch:
  """Device copy of a HostBatch plus outputs and workspace (torch tensors)."""

  def __init__(self, hb: HostBatch, device=None, records: bool | None = None):
    torch = _lib.require_device()
    self.torch = torch
    self.hb = hb
    dev = torch.device(device or "cuda")
    self.device = dev
    f64 = dict(dtype=torch.float64, device=dev)
    u8 = dict(dtype=torch.uint8, device=dev)
    self.inst = torch.from_numpy(hb.inst.view(np.uint8)).to(dev)
    self.order = torch.from_numpy(hb.order).to(dev)
    self.a = torch.empty(hb.a_pool.size, **f64)
    self.p = torch.empty(hb.p_pool.size, **f64)
    self.b = torch.empty(hb.b_pool.size, **f64)
    self.c = torch.empty(hb.c_pool.size, **f64)
    self.x = torch.empty(max(hb.n_total, 1), **f64)
    self.y = torch.empty(max(hb.m_total, 1), **f64)
    self.s = torch.empty(max(hb.m_total, 1), **f64)
    self.results = torch.empty(max(hb.count, 1) * _lib.RESULT_DTYPE.itemsize, **u8)
    self.stats = None
    if records or (records is None and hb.opts.collect_stats):
      self.stats = torch.empty(max(hb.count, 1) * hb.opts.max_iter * _lib.STATS_DOUBLES, **f64)
    self.workspace = torch.empty(hb.workspace_bytes, **u8)
    self._copts = hb.opts.to_c()
    # Pinned staging copies of the inputs for asynchronous host->device copies.
    if hb.pinned:
      self.h_pools = hb.h_pools
    else:
      self.h_pools = [torch.from_numpy(x).pin_memory() for x in
                      (hb.a_pool, hb.p_pool, hb.b_pool, hb.c_pool)]
    self._h_out = None

  def solve_pipelined(self, stream=None) -> None:
    """Packs, copies and launches the batch group by group: each launch group
    is packed on the host, copied to the device and launched on a stream of
    its own, while the host packs the next group; the outputs are complete on
    `stream` when the call returns (no synchronisation).  The host batch must
    have been built with defer=True.

    Groups go in increasing order of their packed bytes (Johnson's rule for a
    two-stage flow shop whose stages are host packing and device solving:
    packing takes less time than solving for every group here, so the
    cheapest packing goes first and the device starts at once, while the
    host packs the big groups behind the running ones)."""
    torch = self.torch
    lib = _lib.load()
    hb = self.hb
    st = stream or torch.cuda.current_stream(self.device)
    ready = torch.cuda.Event()
    ready.record(st)
    streams = _side_streams(torch, self.device, hb.plan.num_groups)
    args_tail = (self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(),
                 self.results.data_ptr(),
                 self.stats.data_ptr() if self.stats is not None else None,
                 self.workspace.data_ptr(), hb.workspace_bytes, ctypes.byref(self._copts))
    done = [None] * hb.plan.num_groups
    self._group_done = done
    for g in hb.launch_order():
      rngs = hb.gather_group(g)
      sg = streams[g]
      sg.wait_event(ready)
      with torch.cuda.stream(sg):
        for dst, src, (lo, hi) in zip((self.a, self.p, self.b, self.c), self.h_pools, rngs):
          if hi > lo:
            dst[lo:hi].copy_(src[lo:hi], non_blocking=True)
      _lib.check(lib.qtqp_dense_batch_solve_group(
          self.inst.data_ptr(), self.order.data_ptr(), ctypes.byref(hb.plan), g,
          self.a.data_ptr(), self.p.data_ptr(), self.b.data_ptr(), self.c.data_ptr(),
          *args_tail, _lib.stream_handle(sg)))
      ev = torch.cuda.Event()
      ev.record(sg)
      done[g] = ev
    hb.gathered = True
    for ev in done:
      st.wait_event(ev)

  def fetch_groups(self):
    """After solve_pipelined: yields (g, results, x, y, s) for each launch
    group as soon as its launch has finished (polling, the other groups may
    still run): the full results array (only group g's entries are final)
    and group g's contiguous output ranges, as numpy arrays owned by the
    caller."""
    torch = self.torch
    hb = self.hb
    copy_stream = _side_streams(torch, self.device, QTQP_COPY_STREAM + 1)[QTQP_COPY_STREAM]
    pending = list(range(hb.plan.num_groups))
    while pending:
      ready = [g for g in pending if self._group_done[g].query()]
      if not ready:
        time.sleep(2e-5)
        continue
      for g in ready:
        pending.remove(g)
        grp = hb.plan.groups[g]
        ids = hb.order[grp.begin:grp.begin + grp.count]
        if not len(ids):
          continue
        n0 = int(hb.inst["n_off"][ids[0]])
        n1 = int(hb.inst["n_off"][ids[-1]] + hb.inst["n"][ids[-1]])
        m0 = int(hb.inst["m_off"][ids[0]])
        m1 = int(hb.inst["m_off"][ids[-1]] + hb.inst["m"][ids[-1]])
        copy_stream.wait_event(self._group_done[g])
        if hb.arena is not None:  # through the arena's pinned buffers into numpy arrays
          nres = (self.results.numel() + 7) // 8
          rb = hb.arena.get("out_res", nres).view(torch.uint8)[:self.results.numel()]
          xb, yb = hb.arena.get("out_x", n1 - n0), hb.arena.get("out_y", m1 - m0)
          sb = hb.arena.get("out_s", m1 - m0)
          with torch.cuda.stream(copy_stream):
            rb.copy_(self.results, non_blocking=True)
            xb.copy_(self.x[n0:n1], non_blocking=True)
            yb.copy_(self.y[m0:m1], non_blocking=True)
            sb.copy_(self.s[m0:m1], non_blocking=True)
          copy_stream.synchronize()
          yield (g, rb.numpy().view(_lib.RESULT_DTYPE)[:hb.count].copy(), n0,
                 xb.numpy().copy(), m0, yb.numpy().copy(), sb.numpy().copy())
          continue
        with torch.cuda.stream(copy_stream):
          res = self.results.to("cpu", non_blocking=True)
          x = self.x[n0:n1].to("cpu", non_blocking=True)
          y = self.y[m0:m1].to("cpu", non_blocking=True)
          sl = self.s[m0:m1].to("cpu", non_blocking=True)
        copy_stream.synchronize()
        yield (g, res.numpy().view(_lib.RESULT_DTYPE)[:hb.count], n0, x.numpy(), m0,
               y.numpy(), sl.numpy())

  def refresh_plan(self) -> None:
    """Re-uploads the descriptors and order and resizes the workspace after
    the host batch was re-planned (HostBatch.replan)."""
    torch = self.torch
    hb = self.hb
    self.inst = torch.from_numpy(hb.inst.view(np.uint8)).to(self.device)
    self.order = torch.from_numpy(hb.order).to(self.device)
    if self.workspace.numel() < hb.workspace_bytes:
      self.workspace = torch.empty(hb.workspace_bytes, dtype=torch.uint8, device=self.device)

  def launch_group(self, g: int, stream=None) -> None:
    """Enqueues launch group g of the plan alone (for timing one group)."""
    hb = self.hb
    full = hb.plan
    one = _lib.BatchPlan()
    ctypes.memmove(ctypes.byref(one), ctypes.byref(full), ctypes.sizeof(one))
    one.num_groups = 1
    one.groups[0] = full.groups[g]
    hb.plan = one
    try:
      self.launch(stream)
    finally:
      hb.plan = full

  def upload(self, stream=None) -> None:
    torch = self.torch
    if not self.hb.gathered:
      self.hb.gather_all()
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip((self.a, self.p, self.b, self.c), self.h_pools):
        dst.copy_(src, non_blocking=True)

  def launch(self, stream=None, start=None) -> None:
    """Enqueues the persistent batch solve on `stream` (no synchronisation).
    start: optional device tensors (x0, y0, s0) laid out like x / y / s,
    starting points that replace the cold start (see start_points)."""
    torch = self.torch
    lib = _lib.load()
    st = stream or torch.cuda.current_stream(self.device)
    hb = self.hb
    args = (self.inst.data_ptr(), self.order.data_ptr(), ctypes.byref(hb.plan),
            self.a.data_ptr(), self.p.data_ptr(), self.b.data_ptr(), self.c.data_ptr(),
            self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(), self.results.data_ptr(),
            self.stats.data_ptr() if self.stats is not None else None,
            self.workspace.data_ptr(), hb.workspace_bytes, ctypes.byref(self._copts))
    if start is None:
      _lib.check(lib.qtqp_dense_batch_solve(*args, _lib.stream_handle(st)))
    else:
      x0, y0, s0 = start
      if (x0.numel() < hb.n_total or y0.numel() < hb.m_total or s0.numel() < hb.m_total):
        raise ValueError("start: pools smaller than the batch's x / y / s")
      _lib.check(lib.qtqp_dense_batch_solve_from(*args, x0.data_ptr(), y0.data_ptr(),
                                                 s0.data_ptr(), _lib.stream_handle(st)))

  def launch_noalloc(self, stream=None) -> None:
    """Enqueues the allocation-free variant: same solve, but its scratch is the
    library's fixed device array instead of this batch's workspace tensor (for
    callers that may not allocate device memory at solve time).  Raises
    QtqpCudaError when the plan needs more scratch than that array holds."""
    torch = self.torch
    lib = _lib.load()
    st = stream or torch.cuda.current_stream(self.device)
    _lib.check(lib.qtqp_dense_batch_solve_noalloc(
        self.inst.data_ptr(), self.order.data_ptr(), ctypes.byref(self.hb.plan),
        self.a.data_ptr(), self.p.data_ptr(), self.b.data_ptr(), self.c.data_ptr(),
        self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(), self.results.data_ptr(),
        self.stats.data_ptr() if self.stats is not None else None, ctypes.byref(self._copts),
        _lib.stream_handle(st)))

  def download(self, stream=None) -> None:
    """Enqueues the device->host copies of the outputs into pinned buffers."""
    torch = self.torch
    if self._h_out is None:
      self._h_out = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                     for t in (self.results, self.x, self.y, self.s)]
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip(self._h_out, (self.results, self.x, self.y, self.s)):
        dst.copy_(src, non_blocking=True)

  @property
  def output_bytes(self) -> int:
    return sum(int(t.numel() * t.element_size()) for t in (self.results, self.x, self.y, self.s))

  def fetch(self):
    """Copies the outputs back, synchronises, and returns (results, x, y, s,
    stats) as numpy arrays owned by the caller."""
    self.download()
    self.torch.cuda.synchronize(self.device)
    res_b, x, y, s = (t.numpy() for t in self._h_out)
    res = res_b.view(_lib.RESULT_DTYPE)[: self.hb.count].copy()
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(self.hb.count, self.hb.opts.max_iter,
                                                _lib.STATS_DOUBLES)
    return (res, x.copy(), y.copy(), s.copy(), stats)


def start_points(hb: HostBatch, problems: Sequence, points: Sequence, shift: float = 0.1):
  """Host pools (x0, y0, s0) of starting points for DeviceBatch.launch.

  points[j]: a Solution (or an (x, y, s) triple) of problems[j] -- typically
  an earlier solve of the same or a nearby QP -- or None for the cold start
  (x = 0, y = s = 1 on the inequality rows).  y and s of a solution sit on the
  cone's boundary, so their inequality rows are moved inside: max(., 0) +
  shift.  Points of a QP whose presolve dropped rows may be given with all
  rows (as Solutions are); the dropped rows are left out.  A point with
  non-finite entries (a certificate) falls back to the cold start.
  """
  if shift <= 0:
    raise ValueError("shift must be positive: the method starts inside the cone")
  x0 = np.zeros(max(hb.n_total, 1))
  y0 = np.zeros(max(hb.m_total, 1))
  s0 = np.zeros(max(hb.m_total, 1))
  for j, (q, pt) in enumerate(zip(problems, points)):
    d = hb.inst[j]
    n0, m0, n, m, z = (int(d[k]) for k in ("n_off", "m_off", "n", "m", "z"))
    y0[m0 + z:m0 + m] = 1.0
    s0[m0 + z:m0 + m] = 1.0
    if pt is None:
      continue
    x, y, sl = (pt.x, pt.y, pt.s) if hasattr(pt, "x") else pt
    x, y, sl = (np.asarray(v, dtype=np.float64) for v in (x, y, sl))
    keep = getattr(getattr(q, "_presolve_state", None), "keep", None)
    if keep is not None and y.shape[0] == keep.shape[0]:
      y, sl = y[keep], sl[keep]
    if x.shape != (n,) or y.shape != (m,) or sl.shape != (m,):
      raise ValueError(f"initial point {j}: shapes {x.shape}, {y.shape}, {sl.shape} do not "
                       f"match the problem's n={n}, m={m}")
    if not (np.all(np.isfinite(x)) and np.all(np.isfinite(y[:z])) and
            np.all(np.isfinite(y[z:])) and np.all(np.isfinite(sl[z:]))):
      continue
    x0[n0:n0 + n] = x
    y0[m0:m0 + z] = y[:z]
    y0[m0 + z:m0 + m] = np.maximum(y[z:], 0.0) + shift
    s0[m0 + z:m0 + m] = np.maximum(sl[z:], 0.0) + shift
  return x0, y0, s0


_SIDE_STREAMS: dict = {}
QTQP_COPY_STREAM = 8  # the side stream after the 8 launch groups' ones: read-backs


def _side_streams(torch, device, count: int):
  """`count` reusable side streams of `device` (created once per device).
  Stream 0 (launch group 0, the costliest instances) has a high priority, as
  the library's own side streams do."""
  key = str(device)
  have = _SIDE_STREAMS.setdefault(key, [])
  while len(have) < count:
    have.append(torch.cuda.Stream(device=device, priority=-1 if not have else 0))
  return have[:count]
