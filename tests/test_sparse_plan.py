"""The symbolic plan of the supernodal factorisation (host code of
libqtqp_cuda, no GPU): the factor it lays out equals a dense Cholesky of the
permuted Gram matrix when the device's numeric phases are replayed in numpy
(tests/sparse_plan_check.py), the update lists are exactly the descendants
with rows in each supernode, the schedule covers every supernode once and
respects the dependencies, and the ordering keeps the fill of a 2D grid near
minimum-degree quality."""

import numpy as np
import pytest
import scipy.sparse as sp

from qtqp_b200 import problems, sparse
from tests import sparse_plan_check as spc


def _gram(a, p, rng):
  m, n = a.shape
  d = rng.uniform(0.5, 2.0, size=m)
  g = (a.T @ sp.diags(d) @ a).toarray() + np.eye(n)
  if p is not None:
    g += p.toarray()
  return g


def _cases():
  rng = np.random.default_rng(11)
  out = []
  for n, m, per_row in ((200, 300, 3), (400, 420, 2), (64, 50, 8), (500, 700, 2)):
    a, _, _, _, p = problems.sparse_feasible(n, m, n // 10, int(rng.integers(1 << 20)),
                                             per_row=per_row)
    out.append((a, p))
  a, _, _, _, p = problems.grid_flow(8)
  out.append((a, p))
  a, _, _, _, _ = problems.sparse_feasible(150, 200, 10, 5, lp=True)
  out.append((a, None))
  return out


@pytest.mark.parametrize("case", range(6))
@pytest.mark.parametrize("ordering", ["amd", "natural"])
def test_plan_factor_equals_dense_cholesky(case, ordering):
  a, p = _cases()[case]
  plan = sparse.SparsePlan(a, p, ordering=ordering)
  n = a.shape[1]
  assert sorted(plan.perm.tolist()) == list(range(n))
  g = _gram(a, p, np.random.default_rng(case))
  gp = g[np.ix_(plan.perm, plan.perm)]
  vals = spc.factor(plan, gp)
  lower = spc.dense_factor(plan, vals)
  np.testing.assert_allclose(lower, np.linalg.cholesky(gp), rtol=0, atol=1e-10)
  v = np.random.default_rng(1).normal(size=n)
  np.testing.assert_allclose(spc.solve(plan, vals, v), np.linalg.solve(gp, v), rtol=1e-9,
                             atol=1e-9)


@pytest.mark.parametrize("case", range(6))
def test_update_lists_and_schedule(case):
  a, p = _cases()[case]
  plan = sparse.SparsePlan(a, p)
  d = plan.desc
  ns = int(d.nsuper)
  first, rowptr, rows = plan.section("first"), plan.section("rowptr"), plan.section("rows")
  colsn = plan.section("colsn")
  assert first[0] == 0 and first[-1] == d.n
  assert np.all(np.diff(first) >= 1) and np.diff(first).max() <= 64
  # Update lists: every (descendant, run of rows in the target's columns).
  expect = {s: [] for s in range(ns)}
  parent = np.full(ns, -1)
  for s in range(ns):
    w = first[s + 1] - first[s]
    r = rows[rowptr[s]:rowptr[s + 1]]
    assert np.array_equal(r[:w], np.arange(first[s], first[s + 1]))
    assert np.all(np.diff(r) > 0)
    if r.size > w:
      parent[s] = colsn[r[w]]
    k = w
    while k < r.size:
      t = colsn[r[k]]
      e = k
      while e < r.size and colsn[r[e]] == t:
        e += 1
      expect[t].append((s, k, e - k))
      k = e
  up, src = plan.section("upd_ptr"), plan.section("upd_src")
  off, cnt = plan.section("upd_off"), plan.section("upd_cnt")
  for s in range(ns):
    got = sorted(zip(src[up[s]:up[s + 1]].tolist(), off[up[s]:up[s + 1]].tolist(),
                     cnt[up[s]:up[s + 1]].tolist()))
    assert got == sorted(expect[s])
  # Schedule: subtrees (contiguous postorder ranges) and top levels cover
  # every supernode once; a top supernode's children run before it.
  seen = np.zeros(ns, dtype=int)
  when = np.full(ns, -1)
  cta_ptr, cta_range = plan.section("cta_ptr"), plan.section("cta_range")
  assert cta_ptr.size == d.blocks + 1
  for q in range(int(cta_ptr[-1])):
    lo, hi = int(cta_range[2 * q]), int(cta_range[2 * q + 1])
    seen[lo:hi + 1] += 1
    when[lo:hi + 1] = -1
    for s in range(lo, hi):  # a subtree: every member's parent is inside, but the root's
      assert lo <= parent[s] <= hi
  top_ptr, top_list = plan.section("top_ptr"), plan.section("top_list")
  for lvl in range(int(d.top_levels)):
    for s in top_list[top_ptr[lvl]:top_ptr[lvl + 1]]:
      seen[s] += 1
      when[s] = lvl
  assert np.all(seen == 1)
  slab = plan.section("top_slab")  # row slabs (64 rows) of the top supernodes, prefix counts
  assert slab[0] == 0 and slab.size == top_list.size + 1
  for q, s in enumerate(top_list):
    assert slab[q + 1] - slab[q] == -(-(rowptr[s + 1] - rowptr[s]) // 64)
  for s in range(ns):
    if parent[s] >= 0 and when[parent[s]] >= 0 and when[s] >= 0:
      assert when[s] < when[parent[s]]
    if parent[s] >= 0 and when[s] >= 0:
      assert when[parent[s]] >= 0  # above a top supernode is only top supernodes


def test_minimum_degree_fill_on_a_grid():
  """The 5-point grid graph (a grid network's incidence rows): minimum degree
  keeps nnz(L) near 31 n at k = 100, against k n for a band ordering."""
  k = 100
  n = k * k
  idx = np.arange(n).reshape(k, k)
  e = ([(idx[i, j], idx[i, j + 1]) for i in range(k) for j in range(k - 1)] +
       [(idx[i, j], idx[i + 1, j]) for i in range(k - 1) for j in range(k)])
  m = len(e)
  a = sp.csc_matrix((np.tile([1.0, -1.0], m), (np.repeat(np.arange(m), 2), np.ravel(e))),
                    shape=(m, n))
  plan = sparse.SparsePlan(a, None)
  assert plan.nnz_l < 40 * n
  assert sparse.SparsePlan(a, None, ordering="natural").nnz_l > 50 * n


def test_analyze_rejects_bad_input():
  a = sp.csc_matrix(np.eye(3))
  bad = sp.csc_matrix((np.ones(1), ([5], [0])), shape=(6, 3))
  from qtqp_b200 import _lib
  with pytest.raises(_lib.QtqpCudaError, match="out of range"):
    sparse.SparsePlan(sp.csc_matrix((bad.data, bad.indices, bad.indptr), shape=(3, 3)), None)
  with pytest.raises(ValueError, match="ordering"):
    sparse.SparsePlan(a, None, ordering="metis")
