"""The MLP oracle's hand-derived backward pass against central finite
differences (CPU only), and the warm-start target encoding."""

import numpy as np

from qtqp_b200 import warmstart
from tests import mlp_oracle


def _params(rng, dim=4, hidden=6, out=5):
  return [rng.normal(size=(dim, hidden)), rng.normal(size=hidden) * 0.1,
          rng.normal(size=(hidden, hidden)), rng.normal(size=hidden) * 0.1,
          rng.normal(size=(hidden, out)), rng.normal(size=out) * 0.1]


def test_backward_matches_finite_differences():
  rng = np.random.default_rng(0)
  params = _params(rng)
  x = rng.normal(size=(7, 4))
  t = rng.normal(size=(7, 5))
  grads = mlp_oracle.gradients(params, x, t)
  h = 1e-6
  for p, g in zip(params, grads):
    flat, gflat = p.reshape(-1), g.reshape(-1)
    for idx in range(flat.size):
      old = flat[idx]
      flat[idx] = old + h
      lp = mlp_oracle.loss(params, x, t)
      flat[idx] = old - h
      lm = mlp_oracle.loss(params, x, t)
      flat[idx] = old
      np.testing.assert_allclose(gflat[idx], (lp - lm) / (2 * h), rtol=1e-5, atol=1e-8)


def test_hinge_backward_matches_finite_differences():
  """The MSE + hinge gradient (the training change that raises warm-start
  acceptance) against central differences, away from the hinge's kink."""
  rng = np.random.default_rng(1)
  params = _params(rng)
  x = rng.normal(size=(7, 4))
  t = rng.normal(size=(7, 5))
  cols = np.array([2, 3, 4])
  zero = rng.normal(size=3) * 0.2
  sign = np.where(t[:, cols] > zero, 1.0, -1.0)
  args = (x, t, cols, zero, sign, 0.7)
  y = mlp_oracle.forward(params, x)[-1]
  kink = np.abs(0.5 - sign * (y[:, cols] - zero))
  assert kink.min() > 1e-3 and np.any(0.5 - sign * (y[:, cols] - zero) > 0)
  grads = mlp_oracle.hinge_gradients(params, *args)
  h = 1e-7
  for p, g in zip(params, grads):
    flat, gflat = p.reshape(-1), g.reshape(-1)
    for idx in range(flat.size):
      old = flat[idx]
      flat[idx] = old + h
      lp = mlp_oracle.hinge_loss(params, *args)
      flat[idx] = old - h
      lm = mlp_oracle.hinge_loss(params, *args)
      flat[idx] = old
      np.testing.assert_allclose(gflat[idx], (lp - lm) / (2 * h), rtol=1e-5, atol=1e-7)
  # With zero weight it is the plain MSE gradient.
  plain = mlp_oracle.gradients(params, x, t)
  for g0, g1 in zip(plain, mlp_oracle.hinge_gradients(params, x, t, cols, zero, sign, 0.0)):
    np.testing.assert_array_equal(g0, g1)


def test_adam_first_step_moves_by_lr():
  p = np.array([1.0, -2.0, 3.0])
  g = np.array([0.5, -0.1, 0.0])
  new, m, v = mlp_oracle.adam_step(p, g, np.zeros(3), np.zeros(3), 1, lr=0.01)
  # Bias-corrected first step: lr * sign(g) (0 where g == 0).
  np.testing.assert_allclose(new, p - 0.01 * np.sign(g), atol=1e-6)


def test_targets_encode_activity_by_sign():
  n, m, z = 2, 4, 1
  x = np.array([[1.0, 2.0]])
  y = np.array([[0.7, 0.0, 1.5, 0.0]])
  s = np.array([[0.0, 0.25, 0.0, 2.0]])
  v = warmstart.targets_from(n, z, x, y, s)
  np.testing.assert_array_equal(v, [[1.0, 2.0, 0.7, -0.25, 1.5, -2.0]])
  xd, yd, act = mlp_oracle.decode(v, np.ones(6), np.zeros(6), n, m, z, 0.0)
  np.testing.assert_array_equal(xd, x)
  np.testing.assert_array_equal(yd, y)
  np.testing.assert_array_equal(act, [[1, 0, 1, 0]])
