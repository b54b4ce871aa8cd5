"""Tensor-core (tcgen05) building blocks of the large dense KKT path against
FP64 numpy: the TF32 split and the Gram product X X^T in plain TF32 and in
the three-product split form."""

import numpy as np
import pytest

from qtqp_b200 import _lib

pytestmark = pytest.mark.gpu


def _split(x):
  import torch
  lib = _lib.load()
  dx = torch.from_numpy(x).cuda()
  hi, lo = torch.empty_like(dx), torch.empty_like(dx)
  _lib.check(lib.qtqp_tc_split_tf32(dx.data_ptr(), dx.numel(), hi.data_ptr(), lo.data_ptr(), 0))
  return hi, lo


def test_split_is_exact_and_hi_is_tf32():
  rng = np.random.default_rng(0)
  x = (rng.normal(size=4099) * 10.0 ** rng.integers(-5, 5, size=4099)).astype(np.float32)
  hi, lo = (t.cpu().numpy() for t in _split(x))
  assert np.all(hi.view(np.uint32) & 0x1FFF == 0)
  np.testing.assert_array_equal(hi + lo, x)
  assert np.all(np.abs(lo) <= np.abs(x) * 2.0 ** -11)


@pytest.mark.parametrize("n,k", [(128, 32), (256, 160), (512, 1024)])
@pytest.mark.parametrize("split", [0, 1])
def test_gram_lower_tiles(n, k, split):
  import torch
  lib = _lib.load()
  rng = np.random.default_rng(n + k)
  x = rng.normal(size=(n, k)).astype(np.float32)
  hi, lo = _split(x)
  c = torch.full((n, n), 7.0, dtype=torch.float32, device="cuda")
  err = torch.zeros(1, dtype=torch.int32, device="cuda")
  for _ in range(2):  # repeated launches give the same tiles
    _lib.check(lib.qtqp_tc_gram_f32(n, k, hi.data_ptr(), lo.data_ptr(), k, c.data_ptr(), n,
                                    split, err.data_ptr(), 0))
  torch.cuda.synchronize()
  assert err.item() == 0
  got = c.cpu().numpy().astype(np.float64)
  xd = x.astype(np.float64)
  want = xd @ xd.T
  nt = n // 128
  scale = np.sqrt(np.outer((xd * xd).sum(1), (xd * xd).sum(1)))  # |x_i| |x_j|
  tol = 4e-5 if split else 2e-3  # relative to |x_i| |x_j| (FP32 accumulation over k)
  for ti in range(nt):
    for tj in range(nt):
      blk = np.s_[ti * 128:(ti + 1) * 128, tj * 128:(tj + 1) * 128]
      if tj > ti:
        assert np.all(got[blk] == 7.0)  # upper tiles untouched
      else:
        rel = np.abs(got[blk] - want[blk]) / scale[blk]
        assert rel.max() < tol, (ti, tj, rel.max())
