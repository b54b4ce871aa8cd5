"""Host packing of the banded batch (CPU only): every instance's A (CSR and
CSC), P, b and c can be read back exactly from the int32/double pools at the
offsets in its descriptor; problems built from the same A and P objects share
one packed copy; the plan orders every instance once and sizes a workspace.
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
