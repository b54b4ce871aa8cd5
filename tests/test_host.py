"""Host-side logic that runs without a GPU: input validation and presolve
(src/qtqp/__init__.py:183-297), the enum surface, the DirectKktSolver driver
(direct.py:112-311) with a CPU test double standing in for the GPU backend,
and the conversion of device stats records into the reference's dicts."""

import numpy as np
import pytest
import scipy.sparse as sp

import qtqp_b200 as qb
from oracle import qtqp_oracle as orc
from qtqp_b200 import batch, direct, problems
from tests import kkt_driver


def test_enum_surface():
  assert qb.LinearSolver.AUTO.value == "auto"
  assert qb.LinearSolver.CUDA.value is direct.CudaDenseSolver
  assert {s.value for s in qb.SolutionStatus} == {
      "solved", "infeasible", "unbounded", "hit_max_iter", "failed", "unfinished"}


def test_validation_errors():
  a, b, c, z, p = problems.feasible(6, 5, 3, 742)
  with pytest.raises(ValueError):
    qb.QTQP(a=a, b=np.zeros(7), c=c, z=z, p=p)
  with pytest.raises(ValueError):
    qb.QTQP(a=a, b=b, c=np.zeros(7), z=z, p=p)
  with pytest.raises(ValueError):
    qb.QTQP(a=a, b=b, c=c, z=z, p=sp.csc_matrix(np.ones((6, 5))))
  with pytest.raises(ValueError):
    qb.QTQP(a=a, b=b, c=c, z=-1, p=p)
  with pytest.raises(ValueError):
    qb.QTQP(a=a, b=b, c=c, z=7, p=p)
  with pytest.raises(TypeError):
    qb.QTQP(a=a.tocsr(), b=b, c=c, z=z, p=p)
  with pytest.raises(TypeError):
    qb.QTQP(a=a, b=b, c=c, z=z, p=p.tocsr())
  with pytest.raises(ValueError, match="symmetric"):
    qb.QTQP(a=sp.eye(2, format="csc"), b=np.ones(2), c=np.zeros(2), z=0,
            p=sp.csc_matrix([[1.0, 2.0], [0.0, 1.0]]))
  with pytest.raises(ValueError, match="finite"):
    qb.QTQP(a=sp.eye(2, format="csc"), b=np.ones(2), c=np.zeros(2), z=0,
            p=sp.csc_matrix([[1.0, np.nan], [np.nan, 1.0]]))
  with pytest.raises(ValueError, match="Equality RHS entries"):
    qb.QTQP(a=sp.eye(3, format="csc"), b=np.array([1.0, np.inf, 3.0]), c=np.zeros(3), z=3)
  with pytest.raises(ValueError, match="effective z == m"):
    qb.QTQP(a=sp.eye(3, format="csc"), b=np.ones(3), c=np.zeros(3), z=3)


def test_presolve_drops_and_restores_rows():
  a, b, c, z, p = problems.feasible(20, 10, 3, 7)
  extra = sp.csc_matrix(np.ones((3, 10)))
  a2 = sp.vstack([a, extra], format="csc")
  b2 = np.concatenate([b, [1e21, np.inf, 1e20]])
  q = qb.QTQP(a=a2, b=b2, c=c, z=z, p=p)
  assert q.m == 20 and q.a.shape == (20, 10)
  y, s = q._postsolve(np.arange(20.0), np.arange(20.0), s_dropped=np.array([7.0, 8.0, 9.0]))
  assert y.shape == (23,) and np.all(y[20:] == 0.0) and np.all(s[20:] == [7, 8, 9])
  with pytest.raises(ValueError, match="effective z == m"):
    qb.QTQP(a=a2, b=np.concatenate([b[:3], np.full(20, 1e21)]), c=c, z=3, p=p)
  with pytest.raises(ValueError, match="Inequality RHS"):
    qb.QTQP(a=a, b=np.concatenate([b[:19], [-np.inf]]), c=c, z=z, p=p)


def test_dense_problem_packing():
  a, b, c, z, p = problems.small_dense_instance(3)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  dp = q.dense_problem()
  np.testing.assert_array_equal(dp.a, a.toarray())
  np.testing.assert_array_equal(dp.p, p.toarray())
  assert qb.QTQP(a=a, b=b, c=c, z=z).dense_problem().p is None


def test_options_validation():
  with pytest.raises(AssertionError):
    batch.SolveOptions(step_size_scale=1.0).validate()
  with pytest.raises(AssertionError):
    batch.SolveOptions(max_iterative_refinement_steps=0).validate()
  with pytest.raises(ValueError):
    batch.SolveOptions(precision="fp16").validate()


def test_diag_data_indices_matches_loop():
  rng = np.random.default_rng(0)
  for fmt in ("csc", "csr"):
    m = sp.random(40, 40, density=0.2, format=fmt, rng=rng) + sp.eye(40, format=fmt)
    m = m.asformat(fmt)
    idx = direct.diag_data_indices(m)
    np.testing.assert_array_equal(m.data[idx], m.diagonal())


class _CpuGram(direct.LinearSolver):
  """CPU test double with the plugin contract (wraps the oracle's backend)."""

  def set_kkt(self, kkt):
    super().set_kkt(kkt)

  def set_dims(self, n, m, z):
    self.n, self.m = n, m

  def factorize(self):
    n = self.n
    up = self._kkt.tocsr()
    a = up[:n, n:].T
    p_up = up[:n, :n]
    p = p_up + p_up.T - sp.diags(p_up.diagonal())
    self.be = orc.DenseGramKkt(a, p)
    self.be.update_diag(self._kkt_diag)
    self.be.factorize()

  def solve(self, rhs):
    return self.be.solve(rhs)

  def format(self):
    return "csr"


def test_direct_kkt_solver_host_driver():
  """DirectKktSolver + a CPU double: the reference's KKT residual criterion."""
  rng = np.random.default_rng(842)
  m, n, z = 150, 100, 10
  a, b, c, _, p = problems.feasible(m, n, z, rng)
  mu = rng.uniform()
  s, y = rng.uniform(size=m), rng.uniform(size=m)
  s[:z] = 0.0
  d = np.concatenate([np.zeros(z), s[z:] / y[z:]])
  kkt = kkt_driver.DirectKktSolver(a=a, p=p, z=z, min_static_regularization=1e-8,
                               max_iterative_refinement_steps=10, atol=1e-12, rtol=1e-12,
                               solver=_CpuGram())
  kkt.update(mu=mu, s=s, y=y)
  sol, st = kkt.solve(rhs=np.concatenate([c, b]), warm_start=np.zeros(n + m))
  assert st["converged"] and st["solves"] >= 1
  np.testing.assert_allclose(p @ sol[:n] + mu * sol[:n] + a.T @ sol[n:], c, atol=1e-10,
                             rtol=1e-10)
  np.testing.assert_allclose(-a @ sol[:n] + (d + mu) * sol[n:], b, atol=1e-10, rtol=1e-10)
  assert (kkt._kkt - sp.triu(kkt._kkt)).nnz == 0


class _ScaledGram(_CpuGram):
  """Returns `scale` times the exact regularised solve: refinement contracts
  by |1 - scale| per step (scale in (0, 2)) or grows (scale outside)."""

  def __init__(self, scale):
    self.scale = scale
    self.freed = 0

  def solve(self, rhs):
    return self.scale * super().solve(rhs)

  def free(self):
    self.freed += 1


class _NanGram(_CpuGram):

  def solve(self, rhs):
    return np.full_like(rhs, np.nan)


def _kkt_case(solver, steps, seed=7):
  rng = np.random.default_rng(seed)
  m, n, z = 30, 20, 4
  a, b, c, _, p = problems.feasible(m, n, z, rng)
  s, y = rng.uniform(0.5, 1.5, size=m), rng.uniform(0.5, 1.5, size=m)
  s[:z] = 0.0
  kkt = kkt_driver.DirectKktSolver(a=a, p=p, z=z, min_static_regularization=1e-8,
                               max_iterative_refinement_steps=steps, atol=1e-12, rtol=1e-12,
                               solver=solver)
  kkt.update(mu=0.3, s=s, y=y)
  return kkt, np.concatenate([c, b])


def test_ir_more_steps_never_worse():
  """More refinement steps give a residual no larger (tests/test_qtqp.py:1977-1999)."""
  finals = []
  for steps in (1, 2, 5, 50):
    kkt, rhs = _kkt_case(_ScaledGram(0.5), steps)
    _, st = kkt.solve(rhs=rhs, warm_start=np.zeros(rhs.size))
    assert st["solves"] <= steps and st["status"] != "stalled"
    finals.append(st["final_residual_norm"])
  assert all(f1 >= f2 for f1, f2 in zip(finals, finals[1:]))
  assert finals[-1] < 1e-10 * max(1.0, np.abs(rhs).max())


def test_ir_stall_rule_stops_a_growing_residual():
  """A step that does not reduce the residual ends refinement as "stalled"
  (direct.py:274-283) and returns the last iterate."""
  kkt, rhs = _kkt_case(_ScaledGram(2.5), 20)
  _, st = kkt.solve(rhs=rhs, warm_start=np.zeros(rhs.size))
  assert st["status"] == "stalled" and not st["converged"] and st["solves"] == 1


def test_ir_nan_raises_value_error():
  """NaNs from the backend raise the reference's ValueError (direct.py:293-294)."""
  kkt, rhs = _kkt_case(_NanGram(), 3)
  with pytest.raises(ValueError, match="Linear solver returned NaNs."):
    kkt.solve(rhs=rhs, warm_start=np.zeros(rhs.size))


def test_free_reaches_the_backend():
  backend = _ScaledGram(1.0)
  kkt, _ = _kkt_case(backend, 2)
  kkt.free()
  assert backend.freed == 1


def test_stats_record_conversion_and_log_line(capsys):
  rec = np.zeros(64)
  rec[:22] = np.arange(22, dtype=float)
  rec[18] = 0  # SOLVED
  for blk in range(3):
    base = 31 + 7 * blk
    rec[base:base + 7] = [2, 1e-13, 1.0, 1e-12, 1 if blk else 2, -1 if blk == 0 else 0, 64]
  d = qb._record_to_dict(rec, True, 0.5)
  assert d["iter"] == 0 and d["status"] == qb.SolutionStatus.SOLVED
  assert d["time"] == 19.5
  assert d["q_lin_sys_stats"]["status"] == "stalled"
  assert "tau_method" not in d["q_lin_sys_stats"]
  assert d["predictor_lin_sys_stats"]["tau_method"] == "quadratic"
  assert d["corrector_lin_sys_stats"]["converged"]
  assert {"complementarity", "std_s_over_y"} <= d.keys()
  qb._log_iteration(d)
  line = capsys.readouterr().out
  assert line.startswith("|    0 |") and " *, 2, 2 |" in line


def test_storage_routing_of_banded_problems():
  """A banded QP solved on its own from n >= BAND_GRID_N goes to the whole
  GPU (partitioned band factorisation); in a batch it stays one per block;
  short horizons stay banded; bands too wide for the partitioned form fall
  back to the one-block path."""
  from qtqp_b200 import band
  a, b, c, z, p = problems.mpc_feasible(20)   # n = 1200, half-bandwidth 99
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.n >= qb.BAND_GRID_N
  assert q.storage_format(single=True) == "band_grid"
  assert q.storage_format() == "band"
  a, b, c, z, p = problems.mpc_feasible(10)   # n = 600 < BAND_GRID_N
  assert qb.QTQP(a=a, b=b, c=c, z=z, p=p).storage_format(single=True) == "band"
  assert band.grid_supported(99, 30000)
  assert not band.grid_supported(band.GRID_MAX_BW + 1, 30000)
  assert not band.grid_supported(99, 150)    # fewer columns than two bands


def test_solve_batch_checks_arguments_before_device_work():
  """solve_batch rejects a bad storage name and warm starts that do not fit
  before it touches a GPU (so these errors are the same with or without one)."""
  import types
  a, b, c, z, p = problems.feasible(12, 8, 2, 3)
  dense_q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  with pytest.raises(ValueError, match="storage must be"):
    qb.solve_batch([dense_q], storage="supernodal")
  model = types.SimpleNamespace(n=dense_q.n, m=dense_q.m)
  with pytest.raises(ValueError, match="banded path"):
    qb.solve_batch([dense_q], storage="dense", warm_start=(model, np.zeros((1, 32))))
  a, b, c, z, p = problems.mpc_feasible(4)
  band_q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  wrong = types.SimpleNamespace(n=band_q.n + 1, m=band_q.m)
  with pytest.raises(ValueError, match="model's"):
    qb.solve_batch([band_q], storage="band", warm_start=(wrong, np.zeros((1, 32))))


def test_device_errors_map_to_the_reference_exceptions():
  """The error codes of a device solve become the exceptions the reference
  raises (LinAlgError for a failed Cholesky, ValueError for NaNs) and a
  RuntimeError for a grid barrier that gave up."""
  from qtqp_b200 import _lib
  with pytest.raises(np.linalg.LinAlgError):
    qb._raise_device_error(_lib.QTQP_ERR_NOT_SPD)
  with pytest.raises(ValueError, match="NaNs"):
    qb._raise_device_error(_lib.QTQP_ERR_NAN)
  with pytest.raises(RuntimeError, match="timed out"):
    qb._raise_device_error(_lib.QTQP_ERR_TIMEOUT)


def _shuffled_mpc(horizon, seed=0):
  a, b, c, z, p = problems.mpc_feasible(horizon)
  perm = np.random.default_rng(seed).permutation(a.shape[1])
  return sp.csc_matrix(a[:, perm]), b, c[perm], z, sp.csc_matrix(p[perm][:, perm])


def test_band_ordering_of_a_shuffled_banded_qp():
  """A stage-ordered QP with its variables shuffled is not banded as given;
  the reverse Cuthill-McKee ordering of its Gram graph makes it narrow again,
  so it takes the banded path in that ordering, and x maps back."""
  from qtqp_b200 import band
  a, b, c, z, p = _shuffled_mpc(10)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert 4 * (band.gram_bandwidth(a, p) + 1) > q.n
  assert q.storage_format() == "band"
  perm = q.band_permutation()
  assert sorted(perm.tolist()) == list(range(q.n))
  bp = q.band_problem()
  assert 4 * (bp.bw + 1) <= q.n
  np.testing.assert_array_equal(bp.a.toarray(), a.toarray()[:, perm])
  np.testing.assert_array_equal(bp.c, c[perm])
  x = np.arange(q.n, dtype=float)
  np.testing.assert_array_equal(qb._unpermute(q, x[perm]), x)
  # the oracle on the band-ordered QP, mapped back, is the QP's own solution
  r_band = orc.solve(bp.a, bp.b, bp.c, bp.z, bp.p, backend="superlu")
  r_orig = orc.solve(a, b, c, z, p, backend="superlu")
  assert r_band.status == r_orig.status == "solved"
  np.testing.assert_allclose(qb._unpermute(q, r_band.x), r_orig.x, atol=1e-8)


def test_dense_and_naturally_banded_qps_keep_their_paths():
  a, b, c, z, p = problems.sparse_qp_n200()
  assert qb.QTQP(a=a, b=b, c=c, z=z, p=p).storage_format() == "dense"
  a, b, c, z, p = problems.mpc_feasible(10)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format() == "band" and q.band_permutation() is None


def test_symmetry_check_of_full_csc_matches_the_sparse_difference():
  """The blocked check of a CSC matrix storing all n x n entries gives the
  reference's max |P - P^T| (__init__.py:240-245), including the rejection."""
  from qtqp_b200 import _max_asymmetry
  rng = np.random.default_rng(4)
  for n in (1, 2, 3, 7, 255, 256, 257, 600):
    m = rng.normal(size=(n, n))
    s = m + m.T
    bad = s.copy()
    bad[rng.integers(n), rng.integers(n)] += 1e-6
    for x in (s, bad):
      xc = sp.csc_matrix(x)
      assert xc.nnz == n * n
      d = xc - xc.T
      ref = float(np.max(np.abs(d.data), initial=0.0)) if d.nnz else 0.0
      assert _max_asymmetry(xc) == pytest.approx(ref, abs=1e-15)
  a = sp.csc_matrix(rng.normal(size=(6, 4)))
  p = np.eye(4)
  p[0, 3] = 1e-9
  with pytest.raises(ValueError, match="symmetric"):
    qb.QTQP(a=a, b=np.ones(6), c=np.zeros(4), z=1, p=sp.csc_matrix(p))


def test_storage_of_dense_qps_is_decided_from_entry_counts():
  """A row of A with more than n/4 entries (or a column of P with more than
  n/2 - 1) rules out every banded ordering; the routing then skips the
  bandwidth and ordering passes."""
  from qtqp_b200 import band
  a, b, c, z, p = problems.large_dense(n=256, m=512, z=64, rank=8)
  assert band.wide_by_counts(sp.csc_matrix(a), sp.csc_matrix(p), 256)
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p))
  assert q.storage_format(single=True) == ("large" if 256 >= qb.LARGE_N_SINGLE else "dense")
  a, b, c, z, p = problems.mpc_feasible(10)
  assert not band.wide_by_counts(a, p, a.shape[1])
  wide_p = sp.csc_matrix(np.ones((8, 8)))
  assert band.wide_by_counts(sp.csc_matrix((3, 8)), wide_p, 8)
  # Counts never exceed what the bandwidth itself implies.
  rng = np.random.default_rng(2)
  for _ in range(20):
    n = int(rng.integers(4, 40))
    a = sp.random(int(rng.integers(1, 60)), n, density=float(rng.uniform(0.02, 0.5)),
                  format="csc", random_state=rng)
    dense = a.toarray() != 0
    spans = [np.flatnonzero(r).max() - np.flatnonzero(r).min() for r in dense if r.any()]
    assert band.gram_bandwidth(a, None) == (max(spans) if spans else 0)
    if band.wide_by_counts(a, None, n):
      assert 4 * (band.gram_bandwidth(a, None) + 1) > n


def test_storage_routing_of_sparse_problems():
  """A grid network's QP solved on its own goes to the supernodal path when
  its band is too wide for the partitioned band path (in a batch it stays
  banded); a random sparse QP whose factor fills 25 % of a dense one stays
  dense; a long MPC horizon keeps the partitioned band path."""
  a, b, c, z, p = problems.grid_flow(32)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.sparse_plan().fill_fraction() < qb.SPARSE_FILL
  assert q.storage_format(single=True) == "sparse"
  assert q.storage_format() == "band"
  a, b, c, z, p = problems.sparse_feasible(1200, 1300, 100, 9)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.storage_format(single=True) == "large"
  a, b, c, z, p = problems.mpc_feasible(30)
  assert qb.QTQP(a=a, b=b, c=c, z=z, p=p).storage_format(single=True) == "band_grid"


def test_one_size_instances_are_dense_csc_and_solvable():
  """problems.small_dense_instance_n (the per-size batches of the phase
  reporter): m = 2n, z = n // 4, every entry of A and P stored in CSC order
  (so a batch packs them in place), and the oracle solves them."""
  for n in (8, 13):
    a, b, c, z, p = problems.small_dense_instance_n(n, 0)
    assert a.shape == (2 * n, n) and p.shape == (n, n) and z == n // 4
    assert a.format == "csc" and a.nnz == 2 * n * n and p.nnz == n * n
    again = problems.small_dense_instance_n(n, 0)
    np.testing.assert_array_equal(again[0].toarray(), a.toarray())
    r = orc.solve(a.toarray(), b, c, z, p.toarray())
    assert r.status == "solved"
