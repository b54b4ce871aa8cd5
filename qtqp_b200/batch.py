"""Device-resident batched solve of dense QPs through the C-ABI.

A batch is packed once into flat pools (row-major A and P per instance, b, c),
planned by the library (processing order, launch shape, workspace), copied to
the device, and solved by one persistent launch of
``qtqp_dense_batch_solve``: one thread block runs one QP's whole interior-point
method (the device counterpart of ``QTQP._solve_impl``,
src/qtqp/__init__.py:351-614 of the reference).
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Sequence

import numpy as np

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
    if self.precision not in ("fp64", "mixed"):
      raise ValueError(f"precision must be 'fp64' or 'mixed', got {self.precision!r}")

  def to_c(self) -> _lib.Options:
    return _lib.Options(
        self.atol, self.rtol, self.atol_infeas, self.rtol_infeas,
        self.step_size_scale, self.min_static_regularization,
        self.linear_solver_atol, self.linear_solver_rtol, int(self.max_iter),
        int(self.max_iterative_refinement_steps), int(bool(self.equilibrate)),
        _lib.PREC_FP64 if self.precision == "fp64" else _lib.PREC_MIXED,
        int(bool(self.collect_stats)), int(self.tau_mode), int(self.warm_corrections))


@dataclasses.dataclass
class DenseProblem:
  """One presolved QP in dense form: A (m x n), P (n x n) or None, b, c, z."""

  a: np.ndarray
  b: np.ndarray
  c: np.ndarray
  z: int
  p: np.ndarray | None = None


class HostBatch:
  """Packed host pools of a batch (pinned when torch is available)."""

  def __init__(self, problems: Sequence[DenseProblem], opts: SolveOptions,
               block_threads: int = 0, smem_bytes: int = 0):
    lib = _lib.load()
    count = len(problems)
    self.count = count
    inst = np.zeros(count, dtype=_lib.INSTANCE_DTYPE)
    a_off = p_off = n_off = m_off = 0
    for i, pr in enumerate(problems):
      m, n = pr.a.shape
      inst[i]["n"], inst[i]["m"], inst[i]["z"] = n, m, pr.z
      inst[i]["has_p"] = int(pr.p is not None and np.any(pr.p != 0))
      inst[i]["a_off"], inst[i]["p_off"] = a_off, p_off
      inst[i]["n_off"], inst[i]["m_off"] = n_off, m_off
      inst[i]["st_off"] = i * opts.max_iter
      a_off += m * n
      p_off += n * n if inst[i]["has_p"] else 0
      n_off += n
      m_off += m
    self.a_pool = np.empty(max(a_off, 1))
    self.p_pool = np.zeros(max(p_off, 1))
    self.b_pool = np.empty(max(m_off, 1))
    self.c_pool = np.empty(max(n_off, 1))
    for i, pr in enumerate(problems):
      d = inst[i]
      m, n = int(d["m"]), int(d["n"])
      self.a_pool[d["a_off"]:d["a_off"] + m * n] = np.ascontiguousarray(pr.a, np.float64).ravel()
      if d["has_p"]:
        self.p_pool[d["p_off"]:d["p_off"] + n * n] = np.ascontiguousarray(
            pr.p, np.float64).ravel()
      self.b_pool[d["m_off"]:d["m_off"] + m] = pr.b
      self.c_pool[d["n_off"]:d["n_off"] + n] = pr.c
    self.n_total, self.m_total = n_off, m_off
    order = np.zeros(max(count, 1), dtype=np.int32)
    plan = _lib.BatchPlan()
    copts = opts.to_c()
    _lib.check(lib.qtqp_dense_batch_plan(inst.ctypes.data, count, ctypes.byref(copts),
                                         order.ctypes.data, block_threads, smem_bytes,
                                         ctypes.byref(plan)))
    self.inst, self.order, self.plan = inst, order, plan
    self.workspace_bytes = int(plan.workspace_bytes)
    self.opts = opts

  @property
  def groups(self):
    """(begin, count, block_threads, smem_bytes) of each launch group."""
    return [(g.begin, g.count, g.block_threads, g.smem_bytes)
            for g in self.plan.groups[:self.plan.num_groups]]

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
    # Pinned staging copies of the inputs for end-to-end (host->device) use.
    self.h_pools = [torch.from_numpy(x).pin_memory() for x in
                    (hb.a_pool, hb.p_pool, hb.b_pool, hb.c_pool)]

  def upload(self, stream=None) -> None:
    torch = self.torch
    with torch.cuda.stream(stream or torch.cuda.current_stream(self.device)):
      for dst, src in zip((self.a, self.p, self.b, self.c), self.h_pools):
        dst.copy_(src, non_blocking=True)

  def launch(self, stream=None) -> None:
    """Enqueues the persistent batch solve on `stream` (no synchronisation)."""
    torch = self.torch
    lib = _lib.load()
    st = stream or torch.cuda.current_stream(self.device)
    hb = self.hb
    _lib.check(lib.qtqp_dense_batch_solve(
        self.inst.data_ptr(), self.order.data_ptr(), ctypes.byref(hb.plan),
        self.a.data_ptr(), self.p.data_ptr(), self.b.data_ptr(), self.c.data_ptr(),
        self.x.data_ptr(), self.y.data_ptr(), self.s.data_ptr(), self.results.data_ptr(),
        self.stats.data_ptr() if self.stats is not None else None,
        self.workspace.data_ptr(), hb.workspace_bytes, ctypes.byref(self._copts),
        _lib.stream_handle(st)))

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

  def fetch(self):
    """Synchronises and returns (results, x, y, s, stats) as numpy arrays."""
    self.torch.cuda.synchronize(self.device)
    res = self.results.cpu().numpy().view(_lib.RESULT_DTYPE)[: self.hb.count]
    stats = None
    if self.stats is not None:
      stats = self.stats.cpu().numpy().reshape(self.hb.count, self.hb.opts.max_iter,
                                                _lib.STATS_DOUBLES)
    return (res, self.x.cpu().numpy(), self.y.cpu().numpy(), self.s.cpu().numpy(), stats)
