"""Host packing of the batches (CPU only).  Banded batch: every instance's A
(CSR and CSC), P, b and c read back exactly from the int32/double pools at the
offsets in its descriptor; problems built from the same A and P objects share
one packed copy; the plan orders every instance once and sizes a workspace.
Dense batch: A, P, b and c read back exactly from the column-major pools.
"""

import numpy as np
import scipy.sparse as sp

from qtqp_b200 import band, problems
from qtqp_b200.batch import SolveOptions


def _unpack_csr(ipool, vpool, ptr, idx, val, rows, cols):
  indptr = ipool[ptr:ptr + rows + 1].astype(np.int64)
  nnz = int(indptr[-1])
  return sp.csr_matrix((vpool[val:val + nnz], ipool[idx:idx + nnz], indptr),
                       shape=(rows, cols))


def _batch():
  fam = problems.parametric_mpc_family(count=3, horizon=6)
  shared = [problems.parametric_mpc_instance(fam, i) for i in range(3)]
  other = problems.mpc_feasible(4, nx=4, nu=2)
  qps = shared + [other]
  bps = [band.BandProblem(a, b, c, z, p) for a, b, c, z, p in qps]
  return qps, band.HostBandBatch(bps, SolveOptions())


def test_pools_read_back_every_instance():
  qps, hb = _batch()
  for i, (a, b, c, z, p) in enumerate(qps):
    d = hb.inst[i]
    m, n = a.shape
    assert (int(d["n"]), int(d["m"]), int(d["z"])) == (n, m, z)
    a_csr = _unpack_csr(hb.ipool, hb.vpool, int(d["a_ptr"]), int(d["a_idx"]),
                        int(d["a_val"]), m, n)
    assert abs(a_csr - sp.csr_matrix(a)).max() == 0.0
    at_csr = _unpack_csr(hb.ipool, hb.vpool, int(d["at_ptr"]), int(d["at_idx"]),
                         int(d["at_val"]), n, m)
    assert abs(at_csr - sp.csr_matrix(a).T).max() == 0.0
    assert int(d["has_p"]) == 1
    p_csr = _unpack_csr(hb.ipool, hb.vpool, int(d["p_ptr"]), int(d["p_idx"]),
                        int(d["p_val"]), n, n)
    assert abs(p_csr - sp.csr_matrix(p)).max() == 0.0
    n0, m0 = int(d["n_off"]), int(d["m_off"])
    np.testing.assert_array_equal(hb.b_pool[m0:m0 + m], b)
    np.testing.assert_array_equal(hb.c_pool[n0:n0 + n], c)
    assert int(d["bw"]) == band.gram_bandwidth(a, p)


def test_shared_structure_is_packed_once():
  qps, hb = _batch()
  keys = ("a_ptr", "a_idx", "a_val", "at_ptr", "at_idx", "at_val", "p_ptr", "p_idx", "p_val")
  first = [int(hb.inst[0][k]) for k in keys]
  for i in (1, 2):
    assert [int(hb.inst[i][k]) for k in keys] == first
  assert [int(hb.inst[3][k]) for k in keys] != first
  a0, a3 = qps[0][0], qps[3][0]
  nnz = 2 * (a0.nnz + a3.nnz) + qps[0][4].nnz + qps[3][4].nnz
  assert hb.vpool.size == nnz  # A (CSR + CSC) and P of the two structures, once each


def test_plan_orders_each_instance_once():
  _, hb = _batch()
  assert sorted(hb.order[:hb.count].tolist()) == list(range(hb.count))
  assert hb.workspace_bytes > 0
  assert hb.n_total == sum(int(d["n"]) for d in hb.inst)
  assert hb.m_total == sum(int(d["m"]) for d in hb.inst)


def test_dense_pools_read_back_every_instance():
  """The dense batch's pools (A m x n and P n x n column-major per instance;
  an LP or an all-zero P packs no P) read back exactly at each descriptor's
  offsets, from DenseProblems and from QTQP objects alike; a QTQP whose CSC
  matrices store every entry is packed from its value arrays in place."""
  import qtqp_b200 as qb
  from qtqp_b200 import batch
  probs, qps = [], []
  for i in range(6):
    a, b, c, z, p = problems.small_dense_instance(i)
    if i == 4:  # a sparse A (not every entry stored) packs through a dense copy
      a = sp.csc_matrix(np.where(np.abs(a.toarray()) > 0.5, a.toarray(), 0.0))
    probs.append(batch.DenseProblem(a.toarray(), b, c, z, p.toarray() if i != 2 else None))
    qps.append(qb.QTQP(a=a, b=b, c=c, z=z, p=p if i != 2 else None))
  for src in (probs, qps):
    hb = batch.HostBatch(src, SolveOptions())
    for i, pr in enumerate(probs):
      d = hb.inst[i]
      m, n = pr.a.shape
      a0, p0 = int(d["a_off"]), int(d["p_off"])
      np.testing.assert_array_equal(hb.a_pool[a0:a0 + m * n].reshape(n, m).T, pr.a)
      assert int(d["has_p"]) == (pr.p is not None)
      if pr.p is not None:
        np.testing.assert_array_equal(hb.p_pool[p0:p0 + n * n].reshape(n, n).T, pr.p)
      m0, n0 = int(d["m_off"]), int(d["n_off"])
      np.testing.assert_array_equal(hb.b_pool[m0:m0 + m], pr.b)
      np.testing.assert_array_equal(hb.c_pool[n0:n0 + n], pr.c)
    assert hb.p_pool.size == sum(p.a.shape[1] ** 2 for p in probs if p.p is not None)
  assert all(getattr(q, "_dense_pack", None) is not None for i, q in enumerate(qps) if i != 4)
  assert getattr(qps[4], "_dense_pack", None) is None
