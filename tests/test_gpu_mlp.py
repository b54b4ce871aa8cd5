"""The warm-start MLP kernels against the numpy oracle, and the learned warm
start end to end on a small parametric MPC family: identical statuses to the
plain method, every accepted point passes the termination test, and the
warm-started batch needs fewer IPM iterations."""

import numpy as np
import pytest

import qtqp_b200 as qb
from qtqp_b200 import _lib, band, batch, problems, warmstart
from tests import kkt_checks, mlp_oracle

pytestmark = pytest.mark.gpu

F32_RTOL = 2e-4  # FP32 kernels vs the FP64 oracle
WARM_CORRECTIONS = 8  # active-set corrections after the first reduced solve


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_gemm_all_transposes(ta, tb):
  import torch
  lib = _lib.load()
  rng = np.random.default_rng(ta * 2 + tb)
  m, n, k = 67, 130, 45
  a = rng.normal(size=(k, m) if ta else (m, k)).astype(np.float32)
  b = rng.normal(size=(n, k) if tb else (k, n)).astype(np.float32)
  bias = rng.normal(size=n).astype(np.float32)
  c0 = rng.normal(size=(m, n)).astype(np.float32)
  da, db_, dbias = (torch.from_numpy(v).cuda() for v in (a, b, bias))
  dc = torch.from_numpy(c0).cuda()
  _lib.check(lib.qtqp_mlp_gemm(m, n, k, 1.5, da.data_ptr(), a.shape[1], ta, db_.data_ptr(),
                               b.shape[1], tb, 0.5, dc.data_ptr(), n, dbias.data_ptr(), 1, 0))
  ref = np.maximum(1.5 * ((a.T if ta else a).astype(np.float64) @
                          (b.T if tb else b).astype(np.float64)) + 0.5 * c0 + bias, 0.0)
  np.testing.assert_allclose(dc.cpu().numpy(), ref, rtol=F32_RTOL, atol=1e-4)


def test_gradients_and_adam_match_oracle():
  import torch
  net = warmstart.WarmStartMLP(dim=5, n=4, m=3, z=1, hidden=16, seed=3)
  rng = np.random.default_rng(1)
  x = rng.normal(size=(9, 5)).astype(np.float32)
  t = rng.normal(size=(9, 7)).astype(np.float32)
  xb, tb = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
  loss = torch.zeros(1, dtype=torch.float64, device="cuda")
  for _ in range(2):  # the loss is overwritten, not accumulated
    net.gradients(xb, tb, 9, loss_buf=loss)
  params = [p.astype(np.float64) for p in net.params_host()]
  want = mlp_oracle.gradients(params, x.astype(np.float64), t.astype(np.float64))
  for g, w in zip(net.grads, want):
    np.testing.assert_allclose(g.cpu().numpy(), w, rtol=1e-3, atol=1e-5)
  np.testing.assert_allclose(loss.item() / t.size, mlp_oracle.loss(params, x, t), rtol=1e-4)
  p0 = net.params[0].clone()
  g0 = net.grads[0].clone()
  _lib.check(net.lib.qtqp_mlp_adam(p0.data_ptr(), g0.data_ptr(), net.adam_m[0].data_ptr(),
                                   net.adam_v[0].data_ptr(), p0.numel(), 1e-3, 0.9, 0.999, 1e-8,
                                   1, 0))
  want_p, _, _ = mlp_oracle.adam_step(params[0], g0.cpu().numpy().astype(np.float64),
                                      np.zeros_like(params[0]), np.zeros_like(params[0]), 1)
  np.testing.assert_allclose(p0.cpu().numpy(), want_p, rtol=1e-5, atol=1e-7)


def test_hinge_gradients_match_oracle():
  """MSE + hinge on the sign of the inequality outputs: the device loss and
  gradients against the FP64 oracle (tests/mlp_oracle.py hinge_gradients)."""
  import torch
  n, m, z, dim, weight, margin = 4, 6, 2, 5, 0.7, 0.5
  net = warmstart.WarmStartMLP(dim=dim, n=n, m=m, z=z, hidden=16, seed=4)
  rng = np.random.default_rng(3)
  raw = rng.normal(size=(40, n + m))
  net.fit_scaling(raw)
  x = rng.normal(size=(9, dim)).astype(np.float32)
  t = ((raw[:9] - net.shift) / net.scale).astype(np.float32)
  zero = net.zero_points()
  xb, tb = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
  loss = torch.zeros(1, dtype=torch.float64, device="cuda")
  net.gradients(xb, tb, 9, loss_buf=loss, hinge_weight=weight, hinge_margin=margin, zero=zero)
  params = [p.astype(np.float64) for p in net.params_host()]
  cols = np.arange(n + z, n + m)
  z64 = zero.cpu().numpy().astype(np.float64)
  sign = np.where(t[:, cols] > z64, 1.0, -1.0)
  want = mlp_oracle.hinge_gradients(params, x.astype(np.float64), t.astype(np.float64), cols,
                                    z64, sign, weight, margin)
  for g, w in zip(net.grads, want):
    np.testing.assert_allclose(g.cpu().numpy(), w, rtol=1e-3, atol=1e-5)
  want_loss = mlp_oracle.hinge_loss(params, x.astype(np.float64), t.astype(np.float64), cols,
                                    z64, sign, weight, margin)
  np.testing.assert_allclose(loss.item() / t.size, want_loss, rtol=1e-4)


@pytest.mark.parametrize("m,n,k", [(300, 256, 32), (64, 11000, 256), (129, 130, 40)])
def test_bf16_tensor_core_gemm(m, n, k):
  """qtqp_mlp_gemm_bf16 (tcgen05, BF16 inputs, FP32 accumulation) against an
  FP64 product of the same BF16-rounded operands, with bias, ReLU and the
  BF16 copy of the output."""
  import torch
  lib = _lib.load()
  rng = np.random.default_rng(m + n + k)
  a = torch.from_numpy(rng.normal(size=(m, k)).astype(np.float32)).cuda().to(torch.bfloat16)
  bt = torch.from_numpy(rng.normal(size=(n, k)).astype(np.float32)).cuda().to(torch.bfloat16)
  bias = torch.from_numpy(rng.normal(size=n).astype(np.float32)).cuda()
  c = torch.empty((m, n), dtype=torch.float32, device="cuda")
  c16 = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
  err = torch.zeros(1, dtype=torch.int32, device="cuda")
  _lib.check(lib.qtqp_mlp_gemm_bf16(m, n, k, a.data_ptr(), bt.data_ptr(), c.data_ptr(), n,
                                    bias.data_ptr(), 1, c16.data_ptr(), n, err.data_ptr(), 0))
  torch.cuda.synchronize()
  assert int(err.item()) == 0
  a64 = a.float().cpu().numpy().astype(np.float64)
  b64 = bt.float().cpu().numpy().astype(np.float64)
  want = np.maximum(a64 @ b64.T + bias.cpu().numpy(), 0.0)
  scale = np.sqrt(k)  # size of a K-term sum of unit products
  np.testing.assert_allclose(c.cpu().numpy(), want, rtol=0, atol=1e-4 * scale + 1e-4)
  np.testing.assert_allclose(c16.float().cpu().numpy(), want, rtol=1e-2, atol=1e-2)


def test_bf16_forward_matches_fp32_forward():
  """The MLP's inference on the tensor cores (BF16) against its FP32 forward
  pass: the same outputs up to BF16 input rounding."""
  import torch
  net = warmstart.WarmStartMLP(dim=32, n=40, m=60, z=10, hidden=256, seed=2)
  x = torch.from_numpy(np.random.default_rng(5).normal(size=(300, 32)).astype(np.float32)).cuda()
  y32 = net._forward(x, 300)[2].cpu().numpy()
  y16 = net._forward_bf16(x, 300).cpu().numpy()
  assert np.max(np.abs(y16 - y32)) <= 3e-2 * max(1.0, np.max(np.abs(y32)))


def test_decode_matches_oracle():
  net = warmstart.WarmStartMLP(dim=3, n=4, m=6, z=2, hidden=8, seed=5)
  net.bf16 = False  # decode is checked exactly against the FP32 forward pass
  rng = np.random.default_rng(2)
  thetas = rng.normal(size=(5, 3))
  targets = rng.normal(size=(5, 10))
  net.fit_scaling(targets)
  net.threshold = 0.05
  wx, wy, act = (t.cpu().numpy() for t in net.predict_device(thetas))
  import torch
  pred = net._forward(torch.from_numpy(thetas.astype(np.float32)).cuda(), 5)[2]
  x, y, a = mlp_oracle.decode(pred.cpu().numpy().astype(np.float64), net.scale, net.shift,
                              4, 6, 2, 0.05)
  np.testing.assert_allclose(wx, x.ravel(), rtol=1e-12)
  np.testing.assert_allclose(wy, y.ravel(), rtol=1e-12)
  np.testing.assert_array_equal(act, a.ravel())


def _family(count, horizon=8):
  fam = problems.parametric_mpc_family(count=count, horizon=horizon)
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in
         (problems.parametric_mpc_instance(fam, i) for i in range(count))]
  return fam[-1], qps


def test_warm_start_with_true_active_set_is_accepted():
  """The solver's own solutions, fed back as the warm start, pass the
  acceptance test; rows whose dual and slack are both at the IPM's tolerance
  (their sign is left open) are settled by the corrections."""
  import torch
  _, qps = _family(32)
  q0 = qps[0]
  n, m, z = q0.n, q0.m, q0.z
  hb = band.HostBandBatch([q.band_problem() for q in qps], batch.SolveOptions(warm_corrections=2))
  plain = band.DeviceBandBatch(hb)
  plain.upload()
  plain.launch()
  r_plain, x, y, s, _ = plain.fetch()
  v = warmstart.targets_from(n, z, x.reshape(32, -1), y.reshape(32, -1), s.reshape(32, -1))
  ineq = np.arange(m) >= z
  yv = np.where(ineq, np.maximum(v[:, n:], 0.0), v[:, n:])
  act = np.where(ineq, v[:, n:] > 0, True).astype(np.uint8)
  warm = tuple(torch.from_numpy(np.ascontiguousarray(t).ravel()).cuda()
               for t in (v[:, :n], yv, act))
  d2 = band.DeviceBandBatch(hb)
  d2.upload()
  d2.launch(warm=warm)
  r_warm, xw, yw, sw, _ = d2.fetch()
  np.testing.assert_array_equal(r_warm["status"], r_plain["status"])
  assert r_warm["warm_started"].sum() == 32
  assert r_warm["iterations"].sum() == 0
  # Both points pass the termination test; the objectives agree to 1e-6.
  for i, q in enumerate(qps):
    xi, yi, si = xw[i * n:(i + 1) * n], yw[i * m:(i + 1) * m], sw[i * m:(i + 1) * m]
    e = kkt_checks.kkt_errors(xi, yi, si, q.a, q.b, q.c, q.p)
    assert e["pres"] < 1e-7 + 1e-8 * e["prel"], e
    assert e["dres"] < 1e-7 + 1e-8 * e["drel"], e
    assert np.min(yi[z:]) >= 0.0 and np.min(si[z:]) >= 0.0
    e0 = kkt_checks.kkt_errors(x[i * n:(i + 1) * n], y[i * m:(i + 1) * m],
                               s[i * m:(i + 1) * m], q.a, q.b, q.c, q.p)
    assert abs(e["pcost"] - e0["pcost"]) <= 1e-6 * max(1.0, abs(e0["pcost"]))


def test_rejected_warm_start_falls_back_to_plain_method():
  """A useless prediction (every row active, zero start) is rejected and the
  plain method gives exactly the plain results."""
  import torch
  _, qps = _family(8)
  q0 = qps[0]
  hb = band.HostBandBatch([q.band_problem() for q in qps], batch.SolveOptions())
  plain = band.DeviceBandBatch(hb)
  plain.upload()
  plain.launch()
  r_plain, xp, yp, sp_, _ = plain.fetch()
  warm = (torch.zeros(8 * q0.n, dtype=torch.float64, device="cuda"),
          torch.zeros(8 * q0.m, dtype=torch.float64, device="cuda"),
          torch.ones(8 * q0.m, dtype=torch.uint8, device="cuda"))
  d2 = band.DeviceBandBatch(hb)
  d2.upload()
  d2.launch(warm=warm)
  r_warm, xw, yw, sw, _ = d2.fetch()
  assert r_warm["warm_started"].sum() == 0
  np.testing.assert_array_equal(r_warm["status"], r_plain["status"])
  np.testing.assert_array_equal(r_warm["iterations"], r_plain["iterations"])
  np.testing.assert_array_equal(xw, xp)
  np.testing.assert_array_equal(yw, yp)


def test_learned_warm_start_on_parametric_family():
  """Train on plain solves of 2048 instances, warm-start 64 held-out ones:
  identical statuses, every accepted point passes the termination test, and
  the warm-started batch needs fewer IPM iterations in total."""
  ntrain, ntest = 2048, 64
  thetas, qps = _family(ntrain + ntest)
  train, test = list(range(ntrain)), list(range(ntrain, ntrain + ntest))
  sols = qb.solve_batch([qps[i] for i in train], storage="band")
  # The family holds a few infeasible instances; train on the solved ones.
  keep = [i for i, s in zip(train, sols) if s.status == qb.SolutionStatus.SOLVED]
  assert len(keep) > 0.99 * ntrain
  sols = [s for s in sols if s.status == qb.SolutionStatus.SOLVED]
  q0 = qps[0]
  targets = warmstart.targets_from(q0.n, q0.z, [s.x for s in sols], [s.y for s in sols],
                                   [s.s for s in sols])
  net = warmstart.WarmStartMLP(dim=thetas.shape[1], n=q0.n, m=q0.m, z=q0.z, seed=0)
  rep = net.train(thetas[keep], targets, epochs=40, batch=64, lr=2e-3)
  assert rep.final_loss < rep.losses[0]
  net.calibrate(thetas[keep], targets)
  test_qps = [qps[i] for i in test]
  opts = batch.SolveOptions(warm_corrections=WARM_CORRECTIONS)
  hb = band.HostBandBatch([q.band_problem() for q in test_qps], opts)
  plain = band.DeviceBandBatch(hb)
  plain.upload()
  plain.launch()
  r_plain, *_ = plain.fetch()
  warm_db = band.DeviceBandBatch(hb)
  warm_db.upload()
  warm_db.launch(warm=net.predict_device(thetas[test]))
  r_warm, *_ = warm_db.fetch()
  np.testing.assert_array_equal(r_warm["status"], r_plain["status"])
  accepted = r_warm["warm_started"] == 1
  assert accepted.sum() > ntest // 2
  assert r_warm["iterations"].sum() < r_plain["iterations"].sum()
  sols_w = qb.solve_batch(test_qps, storage="band", warm_start=(net, thetas[test]),
                          warm_corrections=WARM_CORRECTIONS)
  for q, s in zip(test_qps, sols_w):
    kkt_checks.assert_status_certificate(s, q.a, q.b, q.c, q.p, q.z)
