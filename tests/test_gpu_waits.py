"""The bounded device waits give up and report instead of hanging.

The whole-GPU solves synchronise their blocks with a grid barrier, and their
triangular solves hand blocks over through per-block flags; both waits give
up after a poll limit (the solve then reports QTQP_ERR_TIMEOUT, which
solve_batch raises as RuntimeError).  The tensor-core pipelines wait on
mbarriers with the same kind of limit.  qtqp_wait_selftest makes each wait run
out on purpose with a short limit -- a block that never arrives, an mbarrier
nothing arrives on, a flag nothing sets -- and the tests check the reported
status and that the GPU then solves as before.  Nothing faults.
"""

import pytest
import scipy.sparse as sp

import qtqp_b200 as qb
from qtqp_b200 import _lib, problems

pytestmark = pytest.mark.gpu

SHORT_LIMIT = 1 << 18  # polls: a fraction of a second


def _selftest(mode, blocks=8, skip=3):
  import torch
  lib = _lib.load()
  ws = torch.empty(lib.qtqp_wait_selftest_workspace_bytes(), dtype=torch.uint8, device="cuda")
  status = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
  _lib.check(lib.qtqp_wait_selftest(mode, blocks, skip, SHORT_LIMIT, ws.data_ptr(),
                                    status.data_ptr(),
                                    _lib.stream_handle(torch.cuda.current_stream())))
  torch.cuda.synchronize()
  return int(status.item())


def test_grid_barrier_wait_gives_up_and_the_gpu_stays_usable():
  assert _selftest(0, skip=-1) == _lib.QTQP_OK  # every block arrives
  assert _selftest(0, skip=3) == _lib.QTQP_ERR_TIMEOUT
  assert _selftest(0, skip=0) == _lib.QTQP_ERR_TIMEOUT
  assert _selftest(0, skip=-1) == _lib.QTQP_OK  # the next barrier works again
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in
         (problems.small_dense_instance(i) for i in range(4))]
  assert all(s.status == qb.SolutionStatus.SOLVED for s in qb.solve_batch(qps))


def test_mbarrier_wait_gives_up():
  assert _selftest(1) == _lib.QTQP_ERR_TIMEOUT
  a, b, c, z, p = problems.small_dense_instance(5)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  assert q.solve(verbose=False).status == qb.SolutionStatus.SOLVED


def test_flag_wait_gives_up_and_the_gpu_stays_usable():
  assert _selftest(2, skip=-1) == _lib.QTQP_OK  # every flag is set in turn
  assert _selftest(2, skip=3) == _lib.QTQP_ERR_TIMEOUT
  assert _selftest(2, skip=7) == _lib.QTQP_OK  # the last block: nobody waits on it
  assert _selftest(2, skip=-1) == _lib.QTQP_OK
  a, b, c, z, p = problems.large_dense(n=300, m=600, z=64, rank=16, seed=3)
  q = qb.QTQP(a=sp.csc_matrix(a), b=b, c=c, z=z, p=sp.csc_matrix(p))
  assert qb.solve_batch([q], storage="large")[0].status == qb.SolutionStatus.SOLVED


def test_selftest_arguments_are_checked():
  lib = _lib.load()
  import torch
  status = torch.zeros(1, dtype=torch.int32, device="cuda")
  with pytest.raises(_lib.QtqpCudaError):
    _lib.check(lib.qtqp_wait_selftest(0, 1, 0, SHORT_LIMIT, None, status.data_ptr(), None))
  with pytest.raises(_lib.QtqpCudaError):
    _lib.check(lib.qtqp_wait_selftest(1, 8, 0, 1 << 30, None, status.data_ptr(), None))
  with pytest.raises(_lib.QtqpCudaError):
    _lib.check(lib.qtqp_wait_selftest(3, 8, 0, SHORT_LIMIT, None, status.data_ptr(), None))
