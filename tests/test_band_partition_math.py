"""The partitioned band factorisation of the whole-GPU banded solve, restated
in numpy with the kernel's data flow (qtqp_b200/csrc/band_grid.cuh), checked
against a direct solve.  CPU only: it pins the algebra (interior
eliminations with the separator tail, left spikes, Schur blocks, cyclic
reduction over the separators with D^{-1}, the partitioned solve) for ragged
partitions and any separator count, independently of the device code.
"""

import numpy as np
import pytest


def parts(n, bw, p):
  base, rem = divmod(n - (p - 1) * bw, p)
  lo = [k * (base + bw) + min(k, rem) for k in range(p)]
  li = [base + (1 if k < rem else 0) for k in range(p)]
  return lo, li


def band_chol_range(g, lo, nsub, ne):
  """Eliminates the first ne columns of g[lo:lo+nsub, lo:lo+nsub]; returns
  the factor columns and the Schur complement of the rest."""
  w = g[lo:lo + nsub, lo:lo + nsub].copy()
  l = np.zeros((nsub, ne))
  for k in range(ne):
    d = w[k, k]
    assert d > 0
    l[k:, k] = w[k:, k] / np.sqrt(d)
    w[k + 1:, k + 1:] -= np.outer(l[k + 1:, k], l[k + 1:, k])
  return l, w[ne:, ne:]


def partitioned_factor(g, bw, p):
  n = g.shape[0]
  lo, li = parts(n, bw, p)
  lint, wl, d, q, e = {}, {}, {}, {}, {}
  for k in range(p):
    has_sep = k < p - 1
    l, tail = band_chol_range(g, lo[k], li[k] + (bw if has_sep else 0), li[k])
    lint[k] = l  # rows: the interior, then the separator (W_R^T)
    if has_sep:
      d[k] = tail
    if k >= 1:  # left spike W_L = L_I^{-1} G[I, S_{k-1}]
      gis = g[lo[k]:lo[k] + li[k], lo[k] - bw:lo[k]]
      wl[k] = np.linalg.solve(l[:li[k], :], gis)
      q[k - 1] = wl[k].T @ wl[k]
      if has_sep:
        e[k - 1] = -l[li[k]:, :] @ wl[k]  # -W_R^T W_L, rows of S_k
  # Cyclic reduction over the separators j = 1 .. N (1-based).
  nsep = p - 1
  dd = {j: d[j - 1] - q[j - 1] for j in range(1, nsep + 1)}
  ee = {j: e[j - 1] for j in range(1, nsep)}  # C[j+1, j]
  cs, di, yl, yr, rr = {}, {}, {}, {}, {}
  lev = 0
  while (1 << lev) <= nsep:
    h = 1 << lev
    for j in range(h, nsep + 1, 2 * h):
      di[j] = np.linalg.inv(dd[j])
      if j - h >= 1:
        cl = ee[j - 1] if lev == 0 else cs[j]
        yl[j] = di[j] @ cl
      if j + h <= nsep:
        cr = ee[j] if lev == 0 else cs[j + h]
        rr[j] = cr.copy()
        yr[j] = di[j] @ cr.T
    new_c = {}
    for jp in range(2 * h, nsep + 1, 2 * h):
      jl = jp - h
      dd[jp] = dd[jp] - rr[jl] @ yr[jl]
      if jp - 2 * h >= 1:
        new_c[jp] = -rr[jl] @ yl[jl]
      if jp + h <= nsep:
        jr = jp + h
        cl = ee[jp] if lev == 0 else cs[jr]
        dd[jp] = dd[jp] - cl.T @ yl[jr]
    cs.update(new_c)
    lev += 1
  return dict(lo=lo, li=li, lint=lint, wl=wl, di=di, yl=yl, yr=yr, rr=rr, ee=ee, cs=cs,
              levels=lev, nsep=nsep, p=p)


def partitioned_solve(f, v, bw):
  lo, li, p, nsep = f["lo"], f["li"], f["p"], f["nsep"]
  v = v.astype(float).copy()
  y = {}
  cl = {}
  for k in range(p):  # forward per interior; separator rows get -W_R^T y
    l = f["lint"][k]
    y[k] = np.linalg.solve(l[:li[k], :], v[lo[k]:lo[k] + li[k]])
    if k < p - 1:
      hi = lo[k] + li[k]
      v[hi:hi + bw] -= l[li[k]:, :] @ y[k]
    if k >= 1:
      cl[k - 1] = f["wl"][k].T @ y[k]
  t = {j: v[lo[j - 1] + li[j - 1]:lo[j - 1] + li[j - 1] + bw] - cl[j - 1]
       for j in range(1, nsep + 1)}
  z = {}
  for lev in range(f["levels"]):
    h = 1 << lev
    for j in range(h, nsep + 1, 2 * h):
      z[j] = f["di"][j] @ t[j]
    for jp in range(2 * h, nsep + 1, 2 * h):
      jl = jp - h
      t[jp] = t[jp] - f["rr"][jl] @ z[jl]
      if jp + h <= nsep:
        jr = jp + h
        c = f["ee"][jp] if lev == 0 else f["cs"][jr]
        t[jp] = t[jp] - c.T @ z[jr]
  xs = {}
  for lev in reversed(range(f["levels"])):
    h = 1 << lev
    for j in range(h, nsep + 1, 2 * h):
      r = z[j].copy()
      if j - h >= 1:
        r -= f["yl"][j] @ xs[j - h]
      if j + h <= nsep:
        r -= f["yr"][j] @ xs[j + h]
      xs[j] = r
  x = np.zeros_like(v)
  for j, xj in xs.items():
    hi = lo[j - 1] + li[j - 1]
    x[hi:hi + bw] = xj
  for k in range(p):  # backward per interior with the separators known
    l = f["lint"][k]
    rhs = y[k].copy()
    if k >= 1:
      rhs -= f["wl"][k] @ x[lo[k] - bw:lo[k]]
    if k < p - 1:
      hi = lo[k] + li[k]
      rhs -= l[li[k]:, :].T @ x[hi:hi + bw]
    x[lo[k]:lo[k] + li[k]] = np.linalg.solve(l[:li[k], :].T, rhs)
  return x


def random_band_spd(n, bw, rng):
  m = np.zeros((n, n))
  for i in range(n):
    lo = max(0, i - bw)
    m[i, lo:i + 1] = rng.normal(size=i + 1 - lo)
  g = m @ m.T
  idx = np.arange(n)
  g[np.abs(idx[:, None] - idx[None, :]) > bw] = 0.0
  return g + (2 * bw + 2) * np.eye(n)


@pytest.mark.parametrize("n,bw,p", [(120, 4, 1), (97, 3, 2), (200, 5, 4), (300, 7, 6),
                                    (64, 6, 5), (1000, 9, 32), (800, 3, 100)])
def test_partitioned_solve_matches_direct(n, bw, p):
  rng = np.random.default_rng(n + 7 * bw + p)
  g = random_band_spd(n, bw, rng)
  f = partitioned_factor(g, bw, p)
  b = rng.normal(size=n)
  x = partitioned_solve(f, b, bw)
  assert np.abs(g @ x - b).max() <= 1e-10 * max(1.0, np.abs(b).max())


def test_partition_bounds():
  """Every interior is at least bw long for the largest admissible count
  (n + bw) // (2 bw), the rule of qtqp_band_grid_workspace_bytes."""
  for n, bw in [(30000, 99), (3000, 99), (1794, 9), (1000, 99)]:
    p = min(128, (n + bw) // (2 * bw))
    lo, li = parts(n, bw, p)
    assert min(li) >= bw
    assert lo[-1] + li[-1] == n
