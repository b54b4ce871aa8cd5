"""A numpy restatement of the supernodal factorisation's numeric phases as
the device runs them from a symbolic plan (qtqp_b200.sparse.SparsePlan):
assembly through the Gram entry map, left-looking updates from the update
lists, the diagonal block Cholesky with reciprocal diagonal, and the
forward / backward solves.  Test infrastructure: it checks the plan against
a dense Cholesky of the permuted Gram matrix on the CPU."""

import numpy as np


def factor(plan, g_perm):
  """Factor values (plan layout) of the dense symmetric g_perm (plan order)."""
  first, rowptr, valptr = plan.section("first"), plan.section("rowptr"), plan.section("valptr")
  rows = plan.section("rows")
  upd_ptr, upd_src = plan.section("upd_ptr"), plan.section("upd_src")
  upd_off, upd_cnt = plan.section("upd_off"), plan.section("upd_cnt")
  gcol, grow, gpos = plan.section("gcol"), plan.section("grow"), plan.section("gpos")
  vals = np.zeros(int(plan.desc.nvals))
  vals[gpos] = g_perm[grow, gcol]
  ns = int(plan.desc.nsuper)
  blocks = []
  for s in range(ns):
    f, w = int(first[s]), int(first[s + 1] - first[s])
    nr = int(rowptr[s + 1] - rowptr[s])
    blocks.append((f, w, nr, rows[rowptr[s]:rowptr[s + 1]], int(valptr[s])))
  def block(s):
    f, w, nr, r, v = blocks[s]
    return vals[v:v + nr * w].reshape(w, nr).T  # column-major nr x w view
  for s in range(ns):
    f, w, nr, r, _ = blocks[s]
    ls = block(s)
    for u in range(upd_ptr[s], upd_ptr[s + 1]):
      d, off, cnt = int(upd_src[u]), int(upd_off[u]), int(upd_cnt[u])
      ld = block(d)
      rd = blocks[d][3]
      upd = ld[off:] @ ld[off:off + cnt].T
      pos = np.searchsorted(r, rd[off:])
      cols = rd[off:off + cnt] - f
      ls[np.ix_(pos, cols)] -= upd
    dblk = np.tril(ls[:w, :w])
    lb = np.linalg.cholesky(dblk + np.tril(dblk, -1).T)
    ls[:w, :w] = np.tril(lb, -1) + np.diag(1.0 / np.diag(lb))
    if nr > w:
      ls[w:] = np.linalg.solve(lb, ls[w:].T).T
  return vals


def dense_factor(plan, vals):
  """L as a dense lower-triangular matrix (plan order) from the plan's values."""
  n = int(plan.desc.n)
  first, rowptr, valptr = plan.section("first"), plan.section("rowptr"), plan.section("valptr")
  rows = plan.section("rows")
  L = np.zeros((n, n))
  for s in range(int(plan.desc.nsuper)):
    f, w = int(first[s]), int(first[s + 1] - first[s])
    nr = int(rowptr[s + 1] - rowptr[s])
    r = rows[rowptr[s]:rowptr[s + 1]]
    ls = vals[valptr[s]:valptr[s] + nr * w].reshape(w, nr).T
    blk = ls.copy()
    blk[np.arange(w), np.arange(w)] = 1.0 / blk[np.arange(w), np.arange(w)]
    L[np.ix_(r, np.arange(f, f + w))] = blk
  return np.tril(L)


def solve(plan, vals, v):
  """G^{-1} v with the plan's factor, in the device's supernode order."""
  L = dense_factor(plan, vals)
  import scipy.linalg as sla
  y = sla.solve_triangular(L, v, lower=True)
  return sla.solve_triangular(L.T, y, lower=False)
