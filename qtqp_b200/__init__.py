"""qtqp_b200: the QTQP interior-point hot path, native to NVIDIA B200 (sm_100a).

Drop-in for the reference solver's public API (google-deepmind/qtqp v0.0.5,
src/qtqp/__init__.py):

    sol = qtqp_b200.QTQP(a=a, b=b, c=c, z=z, p=p).solve(
        linear_solver=qtqp_b200.LinearSolver.CUDA)

``LinearSolver.CUDA`` runs the whole interior-point method on the GPU (one
thread block per QP, hand-written CUDA kernels behind a C-ABI); only
validation, presolve/postsolve and result formatting stay on the host.
``solve_batch`` solves many independent QPs in one persistent launch.
"""

from __future__ import annotations

import dataclasses
import enum
import sys
import timeit
from typing import Any, Dict, List, Sequence

import numpy as np
import scipy.sparse as sp

from . import _lib
from . import batch as _batch
from . import direct

__version__ = "0.0.5+b200"

# Dense QPs with at least this many variables are solved one at a time by the
# whole GPU (grid mode) instead of one thread block each; a QP solved on its
# own switches earlier.
LARGE_N = 1024
LARGE_N_SINGLE = 256
# A QP with n >= SPARSE_N whose A has at most 10 % nonzeros and whose
# supernodal factor holds at most SPARSE_FILL of a dense factor's entries gets
# the supernodal factorisation when it is not narrow-banded, or when it is
# solved on its own and its band is too wide for the partitioned band path.
# (Measured on a B200: at 7 % fill the supernodal path takes 0.45-0.72 of the
# whole-GPU dense path's time; at 1.2 % it is 40x faster than the one-block
# banded path.)
SPARSE_N = 256
SPARSE_FILL = 0.10
BAND_GRID_N = 1024  # a banded QP solved on its own from this size: the whole GPU

_HEADER = ("| iter |      pcost |      dcost |     pres |     dres |      gap |"
           "   infeas |       mu |  q, p, c |     time |")
_SEPARA = ("|------|------------|------------|----------|----------|----------|"
           "----------|----------|----------|----------|")


class LinearSolver(enum.Enum):
  """KKT backends (src/qtqp/__init__.py:54-68).

  AUTO resolves to CUDA.  CUDA runs the device-resident loop whose KKT layer is
  the CudaDenseSolver algorithm; the class is also usable on its own as a
  plugin for the reference's DirectKktSolver.  The reference's other members
  name CPU / vendor library backends this build does not ship: solving with
  one raises ImportError, as the reference does when a backend's library is
  not installed.
  """

  AUTO = "auto"
  CUDA = direct.CudaDenseSolver
  ACCELERATE = direct.AccelerateSolver
  SCIPY = direct.ScipySolver
  SCIPY_DENSE = direct.ScipyDenseSolver
  CUPY_DENSE = direct.CupyDenseSolver
  UMFPACK = direct.UmfpackSolver
  PARDISO = direct.MklPardisoSolver
  QDLDL = direct.QdldlSolver
  CHOLMOD = direct.CholModSolver
  CUDSS = direct.CuDssSolver
  EIGEN = direct.EigenSolver
  MUMPS = direct.MumpsSolver


class SolutionStatus(enum.Enum):
  """Possible statuses of the QP solution (src/qtqp/__init__.py:129-137)."""

  SOLVED = "solved"
  INFEASIBLE = "infeasible"
  UNBOUNDED = "unbounded"
  HIT_MAX_ITER = "hit_max_iter"
  FAILED = "failed"
  UNFINISHED = "unfinished"


_STATUS_FROM_CODE = {
    0: SolutionStatus.SOLVED,
    1: SolutionStatus.INFEASIBLE,
    2: SolutionStatus.UNBOUNDED,
    3: SolutionStatus.HIT_MAX_ITER,
    4: SolutionStatus.FAILED,
    5: SolutionStatus.UNFINISHED,
}
_LIN_STATUS = {0: "non-converged", 1: "converged", 2: "stalled"}
_TAU_METHOD = {0: "quadratic", 1: "linearized"}
_FOOTER = {
    SolutionStatus.SOLVED: "Solved",
    SolutionStatus.INFEASIBLE: "Primal infeasible / dual unbounded",
    SolutionStatus.UNBOUNDED: "Dual infeasible / primal unbounded",
    SolutionStatus.HIT_MAX_ITER: "Hit maximum iterations",
    SolutionStatus.FAILED: "Failed to converge",
}


@dataclasses.dataclass(frozen=True)
class Solution:
  """Solution of a QP (src/qtqp/__init__.py:140-156).

  x, y, s: primal/dual/slack solution or infeasibility certificate; stats:
  per-iteration dicts (collect_stats=True); status: SolutionStatus.
  """

  x: np.ndarray
  y: np.ndarray
  s: np.ndarray
  stats: List[Dict[str, Any]]
  status: SolutionStatus


@dataclasses.dataclass(frozen=True)
class _PresolveState:
  keep: np.ndarray
  a_dropped: sp.csc_matrix
  b_dropped: np.ndarray


def _max_asymmetry(p: sp.csc_matrix) -> float:
  """max |P - P^T| (__init__.py:240-245 computes it as a sparse difference).
  A CSC matrix that stores all n x n entries in canonical order holds P^T
  row-major in its data array, compared with its transpose in row blocks;
  anything else takes the sparse difference."""
  n = p.shape[0]
  if p.nnz == n * n and p.has_canonical_format:
    d = p.data.reshape(n, n)  # d[j, i] = P[i, j]
    worst, bs = 0.0, 256  # square blocks: both sides stay in cache
    for r0 in range(0, n, bs):
      for c0 in range(r0, n, bs):
        blk = d[r0:r0 + bs, c0:c0 + bs] - d[c0:c0 + bs, r0:r0 + bs].T
        worst = max(worst, float(np.max(np.abs(blk), initial=0.0)))
    return worst
  asym = p - p.T
  return float(np.max(np.abs(asym.data), initial=0.0)) if asym.nnz else 0.0


class QTQP:
  """Primal-dual interior point method for QPs (src/qtqp/__init__.py:168-307).

    min (1/2) x'Px + c'x  s.t.  Ax + s = b,  s[:z] == 0,  s[z:] >= 0.
  """

  def __init__(self, *, a: sp.csc_matrix, b: np.ndarray, c: np.ndarray, z: int,
               p: sp.csc_matrix | None = None):
    self.m, self.n = a.shape
    self.z = z
    if not sp.isspmatrix_csc(a):
      raise TypeError("Constraint matrix 'a' must be in CSC format.")
    self.a = a
    self.b = np.array(b, dtype=np.float64)
    if self.b.shape != (self.m,):
      raise ValueError(f"b must have shape ({self.m},), got {self.b.shape}")
    self.c = np.array(c, dtype=np.float64)
    if self.c.shape != (self.n,):
      raise ValueError(f"c must have shape ({self.n},), got {self.c.shape}")
    if self.z < 0 or self.z > self.m:
      raise ValueError(f"Number of equality constraints z={self.z} must satisfy "
                       f"0 <= z <= m={self.m}")
    self._presolve()
    if self.z == self.m:
      raise ValueError("effective z == m after presolve; some rows may have been dropped")
    if p is None:
      self.p = sp.csc_matrix((self.n, self.n))
    else:
      if not sp.isspmatrix_csc(p):
        raise TypeError("QP matrix 'p' must be in CSC format.")
      if p.shape != (self.n, self.n):
        raise ValueError(f"p must have shape ({self.n}, {self.n}), got {p.shape}")
      if not np.all(np.isfinite(p.data)):
        raise ValueError("QP matrix 'p' must contain only finite values.")
      if _max_asymmetry(p) > 1e-12:
        raise ValueError("QP matrix 'p' must be symmetric.")
      self.p = p

  def _presolve(self, inf_bound: float = 1e20):
    """Drops inequality rows with b >= inf_bound (__init__.py:248-270)."""
    self._presolve_state = None
    if not np.all(np.isfinite(self.b[:self.z])):
      raise ValueError("Equality RHS entries in 'b' must be finite.")
    ineq_b = self.b[self.z:]
    if np.any(np.isnan(ineq_b) | np.isneginf(ineq_b)):
      raise ValueError("Inequality RHS entries in 'b' must be finite, +inf, or >= inf_bound.")
    drop = np.zeros(self.m, dtype=bool)
    drop[self.z:] = ineq_b >= inf_bound
    if not np.any(drop):
      return
    keep = ~drop
    self._presolve_state = _PresolveState(keep=keep, a_dropped=self.a[drop],
                                          b_dropped=self.b[drop])
    self.a = self.a[keep]
    self.b = self.b[keep]
    self.m = int(keep.sum())

  def _postsolve(self, y, s, y_dropped=0.0, s_dropped=np.nan):
    """Restores the dropped rows (__init__.py:272-290)."""
    if self._presolve_state is None:
      return y, s
    ps = self._presolve_state
    m_full = ps.keep.shape[0]
    y_full = np.empty(m_full)
    s_full = np.empty(m_full)
    y_full[ps.keep], y_full[~ps.keep] = y, y_dropped
    s_full[ps.keep], s_full[~ps.keep] = s, s_dropped
    return y_full, s_full

  def _dropped_slack(self, x):
    ps = self._presolve_state
    return 0.0 if ps is None else ps.b_dropped - ps.a_dropped @ x

  def dense_problem(self) -> _batch.DenseProblem:
    """The presolved QP in the dense form the device solver consumes."""
    p = self.p.toarray() if self.p.nnz else None
    return _batch.DenseProblem(a=self.a.toarray(), b=self.b, c=self.c, z=self.z, p=p)

  def band_problem(self):
    """The presolved QP in the sparse form of the banded device solver, its
    variables in the band ordering (band_permutation) when there is one."""
    from . import band as _band  # pylint: disable=g-import-not-at-top
    perm = self.band_permutation()
    if perm is None:
      return _band.BandProblem(self.a, self.b, self.c, self.z, self.p if self.p.nnz else None)
    a_p, p_p = self._permuted
    return _band.BandProblem(a_p, self.b, self.c[perm], self.z, p_p)

  def band_permutation(self):
    """Ordering of the variables under which P + A^T D A is narrow-banded,
    when the natural one is not: a reverse Cuthill-McKee ordering of the
    Gram matrix's sparsity graph (a fill- and bandwidth-reducing ordering;
    the banded device factorisation then works on the permuted QP, whose x
    is permuted back).  None when the natural ordering is narrow or no
    narrow ordering is found.  Computed once."""
    if not hasattr(self, "_perm"):
      self._perm, self._permuted = None, None
      from . import band as _band  # pylint: disable=g-import-not-at-top
      p = self.p if self.p.nnz else None
      if self.n > 96 and 4 * (_band.gram_bandwidth(self.a, p) + 1) > self.n:
        perm = _band.band_ordering(self.a, p)
        if perm is not None:
          a_p = sp.csc_matrix(self.a[:, perm])
          p_p = sp.csc_matrix(p[perm][:, perm]) if p is not None else None
          if 4 * (_band.gram_bandwidth(a_p, p_p) + 1) <= self.n:
            self._perm, self._permuted = perm, (a_p, p_p)
    return self._perm

  def sparse_plan(self):
    """The symbolic plan of the supernodal factorisation of this QP's Gram
    matrix (qtqp_b200.sparse.SparsePlan: minimum-degree ordering,
    supernodes, schedule).  Computed once."""
    plan = getattr(self, "_sparse", None)
    if plan is None or plan[0] is not self.a or plan[1] is not self.p:
      from . import sparse as _sparse  # pylint: disable=g-import-not-at-top
      plan = (self.a, self.p, _sparse.SparsePlan(self.a, self.p if self.p.nnz else None))
      self._sparse = plan
    return plan[2]

  def storage_format(self, single: bool = False) -> str:
    """'band' when the Gram matrix P + A^T D A is narrow-banded (its
    half-bandwidth at most n/4, in the natural ordering or in the band
    ordering of band_permutation) and n > 96 -- 'band_grid' (the whole GPU,
    partitioned band factorisation) instead for a QP solved on its own with
    n >= BAND_GRID_N and a band narrow enough for it; 'sparse' (the whole GPU,
    supernodal factorisation) for a sparse QP with n >= SPARSE_N whose factor
    stays sparse (sparse_plan) and that is either not banded or banded but
    solved on its own without the partitioned band path; otherwise 'large'
    (the whole GPU on one dense QP) when n >= LARGE_N, or n >= LARGE_N_SINGLE
    for a QP solved on its own; else 'dense' (one thread block per QP)."""
    if self.n <= 96:
      return "dense"
    from . import band as _band  # pylint: disable=g-import-not-at-top
    p = self.p if self.p.nnz else None
    sparse_ok = lambda: (self.n >= SPARSE_N and self.a.nnz <= 0.1 * float(self.m) * self.n and
                         self.sparse_plan().fill_fraction() <= SPARSE_FILL)
    if not _band.wide_by_counts(self.a, p, self.n):  # else no ordering makes it narrow
      bw = _band.gram_bandwidth(self.a, p)
      if 4 * (bw + 1) > self.n and self.band_permutation() is not None:
        a_p, p_p = self._permuted
        bw = _band.gram_bandwidth(a_p, p_p)
      if 4 * (bw + 1) <= self.n:
        if single and self.n >= BAND_GRID_N and _band.grid_supported(bw, self.n):
          return "band_grid"
        if single and sparse_ok():
          return "sparse"
        return "band"
    large = self.n >= (LARGE_N_SINGLE if single else LARGE_N)
    if (single or large) and sparse_ok():
      return "sparse"
    return "large" if large else "dense"

  def solve(self, *, atol: float = 1e-7, rtol: float = 1e-8, atol_infeas: float = 1e-8,
            rtol_infeas: float = 1e-9, max_iter: int = 100, step_size_scale: float = 0.99,
            min_static_regularization: float = 1e-8,
            max_iterative_refinement_steps: int = 20, linear_solver_atol: float = 1e-12,
            linear_solver_rtol: float = 1e-12,
            linear_solver: LinearSolver = LinearSolver.AUTO, verbose: bool = True,
            equilibrate: bool = True, collect_stats: bool = False,
            precision: str = "fp64", initial=None) -> Solution:
    """Solves the QP on the GPU (same keyword arguments as the reference,
    __init__.py:309-326, plus ``precision``: 'fp64' or 'mixed', and
    ``initial``: a starting point -- e.g. the Solution of an earlier solve of
    this or a nearby QP -- for QPs on the dense path; no reference
    counterpart, whose re-solve always starts cold)."""
    opts = _batch.SolveOptions(
        atol=atol, rtol=rtol, atol_infeas=atol_infeas, rtol_infeas=rtol_infeas,
        max_iter=max_iter, step_size_scale=step_size_scale,
        min_static_regularization=min_static_regularization,
        max_iterative_refinement_steps=max_iterative_refinement_steps,
        linear_solver_atol=linear_solver_atol, linear_solver_rtol=linear_solver_rtol,
        equilibrate=equilibrate, collect_stats=collect_stats, precision=precision)
    opts.validate()
    if not isinstance(linear_solver, LinearSolver):
      raise ValueError(f"unsupported linear_solver {linear_solver}")
    if linear_solver not in (LinearSolver.AUTO, LinearSolver.CUDA):
      linear_solver.value()  # raises ImportError: the backend is not shipped
    _lib.require_device()
    start = timeit.default_timer()
    if verbose:
      print(f"| QTQP v{__version__}: m={self.m}, n={self.n}, z={self.z}, "
            f"nnz(A)={self.a.nnz}, nnz(P)={self.p.nnz}, linear_solver=CUDA")
    storage = self.storage_format(single=True)
    if initial is not None and storage != "dense":
      storage = "dense" if self.n < LARGE_N else storage
    out = solve_batch([self], storage=storage, _opts=opts, _verbose=verbose, _start=start,
                      initial=None if initial is None else [initial])[0]
    return out


def _record_to_dict(rec: np.ndarray, collect: bool, t_offset: float) -> Dict[str, Any]:
  """One device stats record -> the reference's per-iteration dict
  (__init__.py:967-1007, direct.py:300-307)."""
  keys = ["iter", "ctx", "bty", "pcost", "dcost", "pres", "dres", "gap", "pinfeas",
          "dinfeas", "dinfeas_a", "dinfeas_p", "mu", "sigma", "alpha", "tau", "norm_x",
          "norm_y", "status", "time", "prelrhs", "drelrhs"]
  d: Dict[str, Any] = {}
  for name, blk in (("q_lin_sys_stats", 0), ("predictor_lin_sys_stats", 1),
                    ("corrector_lin_sys_stats", 2)):
    base = 31 + blk * 7
    lin = {"solves": int(rec[base]), "final_residual_norm": float(rec[base + 1]),
           "rhs_norm": float(rec[base + 2]), "tolerance": float(rec[base + 3]),
           "converged": int(rec[base + 4]) == 1, "status": _LIN_STATUS[int(rec[base + 4])],
           "factor_bits": int(rec[base + 6])}
    if int(rec[base + 5]) >= 0:
      lin["tau_method"] = _TAU_METHOD[int(rec[base + 5])]
    d[name] = lin
  for i, k in enumerate(keys):
    d[k] = float(rec[i])
  d["iter"] = int(rec[0])
  d["status"] = _STATUS_FROM_CODE[int(rec[18])]
  d["time"] = float(rec[19]) + t_offset
  if collect:
    for i, k in enumerate(["complementarity", "norm_s", "max_sy", "min_sy", "std_sy",
                           "max_s_over_y", "min_s_over_y", "mean_s_over_y",
                           "std_s_over_y"]):
      d[k] = float(rec[22 + i])
  return d


def _log_iteration(st: Dict[str, Any]) -> None:
  """The reference's iteration line (__init__.py:1014-1035)."""
  infeas = min(st["pinfeas"], st["dinfeas"])

  def ls(d):
    return " *" if d.get("status") == "stalled" else f"{d.get('solves', 0):2}"

  solves = (f"{ls(st['q_lin_sys_stats'])},{ls(st['predictor_lin_sys_stats'])},"
            f"{ls(st['corrector_lin_sys_stats'])}")
  print(f"| {st['iter']:>4} | {st['pcost']:>10.3e} | {st['dcost']:>10.3e} |"
        f" {st['pres']:>8.2e} | {st['dres']:>8.2e} | {st['gap']:>8.2e} |"
        f" {infeas:>8.2e} | {st['mu']:>8.2e} | {solves:>8} | {st['time']:>8.2e} |")


_TUNING = {}


def _dense_tuning(tuning):
  """The launch-shape table of the dense batch: 'auto' = the autotuner's
  cached table for this GPU model (read once), None = the default plan, or
  an explicit table."""
  if tuning != "auto":
    return tuning
  if "auto" not in _TUNING:
    from . import autotune  # pylint: disable=g-import-not-at-top
    try:
      _TUNING["auto"] = autotune.load()
    except (OSError, ValueError):
      _TUNING["auto"] = None
  return _TUNING["auto"]


def solve_batch(problems: Sequence[QTQP], *, precision: str = "fp64", storage: str = "auto",
                warm_start=None, initial=None, initial_shift: float = 0.1, tuning="auto",
                _opts=None,
                _verbose: bool = False, _start: float | None = None,
                **solve_kwargs) -> List[Solution]:
  """Solves independent QPs in one persistent GPU launch.

  Accepts the keyword arguments of QTQP.solve (verbose defaults to False)
  plus warm_corrections and warm_shift.  storage: 'auto' (per problem,
  QTQP.storage_format), 'dense', 'band', 'large', 'band_grid' or 'sparse'
  (the last three solve one problem at a time on the whole GPU).  warm_start: (WarmStartMLP, thetas) for instances of a parametric
  family, all on the banded path -- each instance first solves the KKT system
  on the predicted active set and keeps that point only if the plain
  termination test passes, else the plain method runs (from the prediction
  when warm_shift > 0).  initial: one starting point per problem (a Solution,
  an (x, y, s) triple, or None for the cold start), e.g. the solutions of an
  earlier call on the same or nearby QPs; its inequality rows are moved
  initial_shift inside the cone (dense storage only).  tuning: launch shapes
  of the dense batch -- 'auto' (the autotuner's cached table for this GPU,
  if any; see qtqp_b200.autotune), None (the library's default plan) or a
  table.  Returns one Solution per problem, in order.
  """
  start = timeit.default_timer() if _start is None else _start
  if _opts is None:
    verbose = solve_kwargs.pop("verbose", False)
    solve_kwargs.pop("linear_solver", None)
    opts = _batch.SolveOptions(precision=precision, **solve_kwargs)
    opts.validate()
  else:
    opts, verbose = _opts, _verbose
  # Arguments are checked before any device work.  Dense and banded problems
  # go to their own device batches; each large problem gets the whole GPU in
  # turn.
  kinds = [q.storage_format() if storage == "auto" else storage for q in problems]
  if any(k not in ("dense", "band", "large", "band_grid", "sparse") for k in kinds):
    raise ValueError("storage must be 'auto', 'dense', 'band', 'large', 'band_grid' or "
                     f"'sparse', got {storage!r}")
  if initial is not None:
    if len(initial) != len(problems):
      raise ValueError(f"initial: {len(initial)} points for {len(problems)} problems")
    if any(k != "dense" for k, pt in zip(kinds, initial) if pt is not None):
      raise ValueError("initial points are supported for dense storage only")
  if warm_start is not None:
    if any(k != "band" for k in kinds):
      raise ValueError("warm_start needs every problem on the banded path")
    model, thetas = warm_start
    if any((q.n, q.m) != (model.n, model.m) for q in problems):
      raise ValueError("warm_start: every problem must have the model's (n, m)")
    if np.asarray(thetas).shape[0] != len(problems):
      raise ValueError(f"warm_start: {np.asarray(thetas).shape[0]} parameter vectors for "
                       f"{len(problems)} problems")
  _lib.require_device()
  records = bool(verbose or opts.collect_stats)
  if problems and initial is None and not records and all(k == "dense" for k in kinds):
    return _solve_dense_streamed(problems, opts, _dense_tuning(tuning))
  per = {}  # kind -> (indices, results, x, y, s, stats, inst)
  where = {}
  t_launch = 0.0
  for i in [i for i, k in enumerate(kinds) if k == "large"]:
    from . import large as _large  # pylint: disable=g-import-not-at-top
    dl = _large.DeviceLarge(problems[i], opts, records=records)
    dl.upload()
    t_launch = timeit.default_timer() - start
    dl.launch()
    res, xp, yp, sp_, st = dl.fetch()
    inst = np.zeros(1, dtype=[("n_off", np.int64), ("m_off", np.int64)])
    where[i] = (res[0], xp, yp, sp_, None if st is None else st[0], inst[0])
  for i in [i for i, k in enumerate(kinds) if k == "band_grid"]:
    from . import band as _band  # pylint: disable=g-import-not-at-top
    hb = _band.HostBandBatch([problems[i].band_problem()], opts)
    dg = _band.DeviceBandGrid(hb, records=records)
    dg.upload()
    t_launch = timeit.default_timer() - start
    dg.launch()
    res, xp, yp, sp_, st = dg.fetch()
    where[i] = (res[0], xp, yp, sp_, None if st is None else st[0], hb.inst[0])
  for i in [i for i, k in enumerate(kinds) if k == "sparse"]:
    from . import sparse as _sparse  # pylint: disable=g-import-not-at-top
    q = problems[i]
    plan = q.sparse_plan()
    dsg = _sparse.DeviceSparseGrid(
        plan.permuted(q.a, q.b, q.c, q.z, q.p if q.p.nnz else None), plan, opts,
        records=records)
    dsg.upload()
    t_launch = timeit.default_timer() - start
    dsg.launch()
    res, xp, yp, sp_, st = dsg.fetch()
    where[i] = (res[0], plan.unpermute(xp[:q.n]), yp, sp_, None if st is None else st[0],
                dsg.pools.inst[0])
  for kind in ("dense", "band"):
    idx = [i for i, k in enumerate(kinds) if k == kind]
    if not idx:
      continue
    if kind == "dense":
      # Packed group by group while earlier groups already solve (below),
      # unless starting points are given.
      hb = _batch.HostBatch([problems[i] for i in idx], opts, pinned=True,
                            tuning=_dense_tuning(tuning), defer=initial is None)
      db = _batch.DeviceBatch(hb, records=records)
    else:
      from . import band as _band  # pylint: disable=g-import-not-at-top
      hb = _band.HostBandBatch([problems[i].band_problem() for i in idx], opts)
      db = _band.DeviceBandBatch(hb, records=records)
    t_launch = timeit.default_timer() - start
    if kind == "dense" and initial is None:
      db.solve_pipelined()
      per[kind] = (idx, *db.fetch(), hb.inst)
      continue
    db.upload()
    if warm_start is not None:
      model, thetas = warm_start
      db.launch(warm=model.predict_device(np.asarray(thetas)))
    elif kind == "dense" and initial is not None:
      import torch  # pylint: disable=g-import-not-at-top
      pools = _batch.start_points(hb, [problems[i] for i in idx], [initial[i] for i in idx],
                                  initial_shift)
      db.launch(start=[torch.from_numpy(v).to(db.device) for v in pools])
    else:
      db.launch()
    per[kind] = (idx, *db.fetch(), hb.inst)
  # Errors first, in problem order (every error code of every batch at once).
  errs = [(i, int(r["error"])) for i, (r, *_) in where.items() if int(r["error"])]
  for kind, (idx, res, *_rest) in per.items():
    bad = np.nonzero(res["error"])[0]
    errs += [(idx[j], int(res["error"][j])) for j in bad]
  if errs:
    _raise_device_error(min(errs)[1])
  out: List[Solution | None] = [None] * len(problems)
  for kind, (idx, res, xp, yp, sp_, st, inst) in per.items():
    ns = inst["n"].tolist()
    ms = inst["m"].tolist()
    n_off = inst["n_off"].tolist()
    m_off = inst["m_off"].tolist()
    codes = res["status"].tolist()
    iters = res["iterations"].tolist()
    for j, i in enumerate(idx):
      n0, m0, mj = n_off[j], m_off[j], ms[j]
      x = xp[n0:n0 + ns[j]]
      if kind == "band":
        x = _unpermute(problems[i], x)
      out[i] = _make_solution(problems[i], x, yp[m0:m0 + mj],
                              sp_[m0:m0 + mj], codes[j], iters[j],
                              None if st is None else st[j], opts, verbose, t_launch)
  for i, (r, x_pool, y_pool, s_pool, recs, d) in where.items():
    q = problems[i]
    n0, m0 = int(d["n_off"]), int(d["m_off"])
    x = x_pool[n0:n0 + q.n].copy()
    if kinds[i] == "band_grid":
      x = _unpermute(q, x)
    out[i] = _make_solution(q, x, y_pool[m0:m0 + q.m].copy(),
                            s_pool[m0:m0 + q.m].copy(), int(r["status"]),
                            int(r["iterations"]), recs, opts, verbose, t_launch)
  return out


def _unpermute(q, x_band):
  """x of q from the x of its band-ordered form (band_permutation)."""
  perm = getattr(q, "_perm", None)
  if perm is None:
    return x_band
  x = np.empty_like(x_band)
  x[perm] = x_band
  return x


_ARENA = _batch.PinnedArena()


def _solve_dense_streamed(problems, opts, tuning) -> List[Solution]:
  """All-dense batch without records: packed, copied and launched group by
  group (DeviceBatch.solve_pipelined), and each group's Solutions built as
  soon as its launch finishes, while the others still run."""
  out: List[Solution | None] = [None] * len(problems)
  errs = []
  with _ARENA.lock:  # the pinned pools are reused from call to call
    hb = _batch.HostBatch(problems, opts, pinned=_ARENA, tuning=tuning, defer=True)
    db = _batch.DeviceBatch(hb, records=False)
    db.solve_pipelined()
    n_off, m_off = hb.inst["n_off"], hb.inst["m_off"]
    for g, res, n0, x, m0, y, s in db.fetch_groups():
      grp = hb.plan.groups[g]
      ids = hb.order[grp.begin:grp.begin + grp.count].tolist()
      codes = res["status"][ids].tolist()
      bad = res["error"][ids]
      if bad.any():
        errs += [(ids[k], int(bad[k])) for k in np.nonzero(bad)[0]]
      iters = res["iterations"][ids].tolist()
      for j, i in enumerate(ids):
        q = problems[i]
        a = int(n_off[i]) - n0
        b = int(m_off[i]) - m0
        out[i] = _make_solution(q, x[a:a + q.n], y[b:b + q.m], s[b:b + q.m], codes[j],
                                iters[j], None, opts, False, 0.0)
  if errs:
    _raise_device_error(min(errs)[1])
  return out


def _raise_device_error(code: int) -> None:
  """The reference's exception for a failed solve (direct.py:293-294 for NaNs;
  a failed Cholesky raises numpy's LinAlgError as the dense backend does)."""
  if code == _lib.QTQP_ERR_NOT_SPD:
    raise np.linalg.LinAlgError("Cholesky failed: the KKT Gram matrix is not positive definite")
  if code == _lib.QTQP_ERR_NAN:
    raise ValueError("Linear solver returned NaNs.")
  if code == _lib.QTQP_ERR_TIMEOUT:
    raise RuntimeError("qtqp_b200: a grid barrier of a whole-GPU solve timed out")
  raise RuntimeError(f"qtqp_b200: device error {code}")


_STATUS_LIST = [_STATUS_FROM_CODE[k] for k in range(6)]


def _make_solution(q, x, y, s, code, iters, recs, opts, verbose, t_launch) -> Solution:
  """One Solution from the device outputs of one QP (x, y, s already owned by
  the caller): presolve rows restored (__init__.py:272-297), the per-iteration
  records turned into the reference's dictionaries, the verbose table."""
  status = _STATUS_LIST[code]
  if q._presolve_state is not None:  # pylint: disable=protected-access
    if status == SolutionStatus.INFEASIBLE:
      y, s = q._postsolve(y, s)
    elif status == SolutionStatus.UNBOUNDED:
      y, s = q._postsolve(y, s, y_dropped=np.nan)
    else:
      y, s = q._postsolve(y, s, s_dropped=q._dropped_slack(x))
  st_list: List[Dict[str, Any]] = []
  if recs is not None:
    st_list = [_record_to_dict(recs[k], opts.collect_stats, t_launch) for k in range(iters)]
  if verbose:
    print(f"{_SEPARA}\n{_HEADER}\n{_SEPARA}")
    for st in st_list:
      _log_iteration(st)
    print(f"{_SEPARA}\n| {_FOOTER.get(status, 'Failed to converge')}")
  return Solution(x, y, s, st_list if opts.collect_stats else [], status)


__all__ = ["QTQP", "Solution", "SolutionStatus", "LinearSolver", "solve_batch", "direct",
           "__version__"]
