"""Numpy oracle of the warm-start MLP (theta -> 256 -> 256 -> out, ReLU, MSE;
optionally a hinge term on the sign of the inequality outputs).

Test infrastructure: forward and hand-derived backward in FP64, checked by
finite differences (tests/test_mlp_oracle.py) and used as the reference for
the device kernels (tests/test_gpu_mlp.py).
"""

import numpy as np


def forward(params, x):
  w1, b1, w2, b2, w3, b3 = params
  a1 = x @ w1 + b1
  h1 = np.maximum(a1, 0.0)
  a2 = h1 @ w2 + b2
  h2 = np.maximum(a2, 0.0)
  y = h2 @ w3 + b3
  return a1, h1, a2, h2, y


def loss(params, x, t):
  y = forward(params, x)[-1]
  return float(np.mean((y - t) ** 2))


def gradients(params, x, t):
  """Gradients of mean((y - t)^2) w.r.t. (w1, b1, w2, b2, w3, b3)."""
  fw = forward(params, x)
  y = fw[-1]
  return _backward(params, x, fw, 2.0 * (y - t) / y.size)


def hinge_loss(params, x, t, cols, zero, sign, weight, margin=0.5):
  """mean((y - t)^2) + weight * mean over (batch, cols) of
  relu(margin - sign * (y[:, cols] - zero)): the MSE plus a hinge that pushes
  each inequality output to the side of its decision point (`zero`, the
  standardised value of y - s = 0) given by the target's sign (+1 / -1)."""
  y = forward(params, x)[-1]
  h = np.maximum(margin - sign * (y[:, cols] - zero), 0.0)
  return float(np.mean((y - t) ** 2) + weight * h.mean())


def hinge_gradients(params, x, t, cols, zero, sign, weight, margin=0.5):
  """Gradients of hinge_loss w.r.t. (w1, b1, w2, b2, w3, b3)."""
  fw = forward(params, x)
  y = fw[-1]
  dy = 2.0 * (y - t) / y.size
  active = (margin - sign * (y[:, cols] - zero)) > 0.0
  dy[:, cols] += -weight * sign * active / (y.shape[0] * len(cols))
  return _backward(params, x, fw, dy)


def _backward(params, x, fw, dy):
  _, _, w2, _, w3, _ = params
  a1, h1, a2, h2, _ = fw
  g3 = h2.T @ dy
  gb3 = dy.sum(axis=0)
  dh2 = (dy @ w3.T) * (a2 > 0)
  g2 = h1.T @ dh2
  gb2 = dh2.sum(axis=0)
  dh1 = (dh2 @ w2.T) * (a1 > 0)
  g1 = x.T @ dh1
  gb1 = dh1.sum(axis=0)
  return [g1, gb1, g2, gb2, g3, gb3]


def adam_step(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
  m = b1 * m + (1 - b1) * g
  v = b2 * v + (1 - b2) * g * g
  mh = m / (1 - b1 ** step)
  vh = v / (1 - b2 ** step)
  return p - lr * mh / (np.sqrt(vh) + eps), m, v


def decode(pred, scale, shift, n, m, z, threshold):
  """Warm start (x, y, active) of standardised outputs [x; y_eq; y - s]."""
  v = pred * scale + shift
  x, w = v[:, :n], v[:, n:]
  ineq = np.arange(m) >= z
  y = np.where(ineq, np.maximum(w, 0.0), w)
  active = np.where(ineq, w > threshold, True).astype(np.uint8)
  return x, y, active
