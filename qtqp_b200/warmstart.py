"""Learned warm start for a parametric QP family (no counterpart in the
reference).

A small MLP, theta (dim) -> 256 -> 256 -> v (n + m), is trained on the
solutions that the plain method produces for instances of the family, with
v = [x; y_eq; y_ineq - s_ineq]: on an inequality row at most one of y_i, s_i
is non-zero at a solution, so the sign of the single signed output tells
whether the row is active.  The prediction gives a starting point and an
active set; the device solver then solves the KKT system on that set (with
at most `warm_corrections` primal-dual active-set corrections) and keeps the
result only if the plain termination test passes -- otherwise the plain
method runs, so it is both the fallback and the arbiter.

Training and inference run on the GPU through the library's hand-written
kernels (qtqp_mlp_*: tiled FP32 GEMM with fused bias/ReLU, ReLU backward,
column sums, MSE gradient, the hinge on the sign of the inequality outputs,
Adam, decoding); PyTorch only allocates device memory.  Inference
(predict_device) runs the three layers on the tensor cores in BF16 with FP32
accumulation (qtqp_mlp_gemm_bf16: tcgen05, TMA-fed, fused bias / ReLU and the
next layer's BF16 input); training keeps FP32 weights and gradients.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from . import _lib


@dataclasses.dataclass
class TrainReport:
  epochs: int
  final_loss: float
  losses: list


def targets_from(n: int, z: int, x, y, s) -> np.ndarray:
  """Training targets [x; y_eq; y_ineq - s_ineq] of a batch of solutions
  (x: count x n, y and s: count x m)."""
  x, y, s = (np.atleast_2d(np.asarray(v, dtype=np.float64)) for v in (x, y, s))
  return np.concatenate([x, y[:, :z], y[:, z:] - s[:, z:]], axis=1)


class WarmStartMLP:
  """theta -> standardised [x; y_eq; y_ineq - s_ineq] of the family's
  solutions."""

  def __init__(self, dim: int, n: int, m: int, z: int, hidden: int = 256, seed: int = 0,
               device=None):
    torch = _lib.require_device()
    self.torch, self.lib = torch, _lib.load()
    self.dim, self.n, self.m, self.z, self.hidden = dim, n, m, z, hidden
    self.out = n + m
    dev = torch.device(device or "cuda")
    self.device = dev
    rng = np.random.default_rng(seed)

    def he(fan_in, fan_out):
      return (rng.normal(size=(fan_in, fan_out)) * np.sqrt(2.0 / fan_in)).astype(np.float32)

    shapes = [(dim, hidden), (hidden,), (hidden, hidden), (hidden,), (hidden, self.out),
              (self.out,)]
    init = [he(dim, hidden), np.zeros(hidden, np.float32), he(hidden, hidden),
            np.zeros(hidden, np.float32),
            (he(hidden, self.out) * 0.1).astype(np.float32), np.zeros(self.out, np.float32)]
    self.params = [torch.from_numpy(a).to(dev) for a in init]
    self.grads = [torch.empty(s, dtype=torch.float32, device=dev) for s in shapes]
    self.adam_m = [torch.zeros(s, dtype=torch.float32, device=dev) for s in shapes]
    self.adam_v = [torch.zeros(s, dtype=torch.float32, device=dev) for s in shapes]
    self.step = 0
    self.bf16 = True   # inference on the tensor cores in BF16
    self._wt16 = None  # BF16 W^T copies of the weights (refresh_bf16)
    self.scale = self.shift = None  # standardisation of the targets (FP64)
    self.threshold = 0.0
    self.row_error_rate = None

  # -- kernels ---------------------------------------------------------------
  def _st(self):
    return _lib.stream_handle(self.torch.cuda.current_stream(self.device))

  def _gemm(self, a, b, c, m, n, k, ta=0, tb=0, beta=0.0, bias=None, relu=0):
    lda = a.shape[1] if a.dim() == 2 else 1
    ldb = b.shape[1] if b.dim() == 2 else 1
    _lib.check(self.lib.qtqp_mlp_gemm(m, n, k, 1.0, a.data_ptr(), lda, ta, b.data_ptr(), ldb,
                                      tb, beta, c.data_ptr(), c.shape[1],
                                      bias.data_ptr() if bias is not None else None, relu,
                                      self._st()))

  def _forward(self, x, bs):
    torch = self.torch
    w1, b1, w2, b2, w3, b3 = self.params
    h1 = torch.empty((bs, self.hidden), dtype=torch.float32, device=self.device)
    h2 = torch.empty_like(h1)
    y = torch.empty((bs, self.out), dtype=torch.float32, device=self.device)
    self._gemm(x, w1, h1, bs, self.hidden, self.dim, bias=b1, relu=1)
    self._gemm(h1, w2, h2, bs, self.hidden, self.hidden, bias=b2, relu=1)
    self._gemm(h2, w3, y, bs, self.out, self.hidden, bias=b3)
    return h1, h2, y

  def refresh_bf16(self) -> None:
    """BF16 copies of the weights, transposed (out x in: the K-major B
    operand of the tensor-core GEMM), taken from the FP32 weights."""
    torch = self.torch
    w1, _, w2, _, w3, _ = self.params
    self._wt16 = []
    for w in (w1, w2, w3):
      k, n = w.shape
      wt = torch.empty((n, k), dtype=torch.bfloat16, device=self.device)
      _lib.check(self.lib.qtqp_mlp_to_bf16(w.data_ptr(), k, n, 1, wt.data_ptr(), self._st()))
      self._wt16.append(wt)

  def _gemm_bf16(self, a16, wt16, bias, relu, out_bf16: bool):
    """A (rows x K, BF16) times W (W^T given, N x K) + bias (ReLU) on the
    tensor cores: FP32 output and, when out_bf16, its BF16 copy."""
    torch = self.torch
    rows, k = a16.shape
    n = wt16.shape[0]
    c = torch.empty((rows, n), dtype=torch.float32, device=self.device)
    c16 = torch.empty((rows, n), dtype=torch.bfloat16, device=self.device) if out_bf16 else None
    err = torch.zeros(1, dtype=torch.int32, device=self.device)
    _lib.check(self.lib.qtqp_mlp_gemm_bf16(rows, n, k, a16.data_ptr(), wt16.data_ptr(),
                                           c.data_ptr(), n, bias.data_ptr(), int(relu),
                                           None if c16 is None else c16.data_ptr(), n,
                                           err.data_ptr(), self._st()))
    return c, c16, err

  def _forward_bf16(self, x, bs):
    """The forward pass on the tensor cores (BF16 in, FP32 accumulate);
    returns the FP32 output."""
    torch = self.torch
    if self._wt16 is None:
      self.refresh_bf16()
    _, b1, _, b2, _, b3 = self.params
    k_in = ((self.dim + 7) // 8) * 8  # K of the first layer padded to 8 (16 bytes)
    x16 = torch.zeros((bs, k_in), dtype=torch.bfloat16, device=self.device)
    x16[:, :self.dim] = x.to(torch.bfloat16)
    w1t = self._wt16[0]
    if k_in != self.dim:
      w1p = torch.zeros((w1t.shape[0], k_in), dtype=torch.bfloat16, device=self.device)
      w1p[:, :self.dim] = w1t
      w1t = w1p
    _, h1, e1 = self._gemm_bf16(x16, w1t, b1, True, True)
    _, h2, e2 = self._gemm_bf16(h1, self._wt16[1], b2, True, True)
    y, _, e3 = self._gemm_bf16(h2, self._wt16[2], b3, False, False)
    if int((e1 + e2 + e3).item()) != 0:
      raise RuntimeError("qtqp_mlp_gemm_bf16: a tensor-core pipeline wait timed out")
    return y

  def gradients(self, xb, tb, batch, dy=None, dh1=None, dh2=None, loss_buf=None,
                hinge_weight: float = 0.0, hinge_margin: float = 0.5, zero=None):
    """Forward + backward of the MSE (plus, with hinge_weight > 0, the hinge
    on the sign of each inequality output, zero: the decision points) on one
    minibatch; fills self.grads and loss_buf (a sum over the outputs).
    Returns the network output."""
    torch, lib, st = self.torch, self.lib, self._st()
    f32 = dict(dtype=torch.float32, device=self.device)
    dy = dy if dy is not None else torch.empty((batch, self.out), **f32)
    dh2 = dh2 if dh2 is not None else torch.empty((batch, self.hidden), **f32)
    dh1 = dh1 if dh1 is not None else torch.empty((batch, self.hidden), **f32)
    if loss_buf is None:
      loss_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
    h1, h2, y = self._forward(xb, batch)
    _lib.check(lib.qtqp_mlp_mse_grad(y.data_ptr(), tb.data_ptr(), y.numel(), dy.data_ptr(),
                                     loss_buf.data_ptr(), st))
    if hinge_weight > 0.0 and self.m > self.z:
      _lib.check(lib.qtqp_mlp_hinge_grad(y.data_ptr(), tb.data_ptr(), batch, self.out,
                                         self.n + self.z, zero.data_ptr(), hinge_weight,
                                         hinge_margin, dy.data_ptr(), loss_buf.data_ptr(), st))
    _, _, w2, _, w3, _ = self.params
    g1, gb1, g2, gb2, g3, gb3 = self.grads
    self._gemm(h2, dy, g3, self.hidden, self.out, batch, ta=1)        # dW3 = H2^T dY
    _lib.check(lib.qtqp_mlp_colsum(dy.data_ptr(), batch, self.out, gb3.data_ptr(), st))
    self._gemm(dy, w3, dh2, batch, self.hidden, self.out, tb=1)      # dH2 = dY W3^T
    _lib.check(lib.qtqp_mlp_relu_grad(dh2.data_ptr(), h2.data_ptr(), dh2.numel(), st))
    self._gemm(h1, dh2, g2, self.hidden, self.hidden, batch, ta=1)    # dW2 = H1^T dH2
    _lib.check(lib.qtqp_mlp_colsum(dh2.data_ptr(), batch, self.hidden, gb2.data_ptr(), st))
    self._gemm(dh2, w2, dh1, batch, self.hidden, self.hidden, tb=1)  # dH1 = dH2 W2^T
    _lib.check(lib.qtqp_mlp_relu_grad(dh1.data_ptr(), h1.data_ptr(), dh1.numel(), st))
    self._gemm(xb, dh1, g1, self.dim, self.hidden, batch, ta=1)       # dW1 = X^T dH1
    _lib.check(lib.qtqp_mlp_colsum(dh1.data_ptr(), batch, self.hidden, gb1.data_ptr(), st))
    return y

  # -- public ----------------------------------------------------------------
  def fit_scaling(self, targets: np.ndarray) -> None:
    """Per-coordinate standardisation of the targets."""
    self.shift = targets.mean(axis=0)
    self.scale = np.maximum(targets.std(axis=0), 1e-6)

  def zero_points(self):
    """Standardised value of y_i - s_i = 0 for each inequality output (the
    decision point of its sign), FP32 on the device."""
    c0 = self.n + self.z
    z = (0.0 - self.shift[c0:]) / self.scale[c0:]
    return self.torch.from_numpy(z.astype(np.float32)).to(self.device)

  def train(self, thetas: np.ndarray, targets: np.ndarray, epochs: int = 30, batch: int = 256,
            lr: float = 1e-3, seed: int = 0, hinge_weight: float = 0.0,
            hinge_margin: float = 0.5, cosine: bool = False) -> TrainReport:
    """Adam on the MSE of the standardised targets (plus, with hinge_weight
    > 0, a hinge that pushes each inequality output to the target's side of
    its decision point); all math on the GPU.  cosine: the learning rate
    decays from lr to 0 over the run (cosine schedule).  The mean loss of
    each epoch is read back once per epoch."""
    torch = self.torch
    if self.scale is None:
      self.fit_scaling(targets)
    rng = np.random.default_rng(seed)
    # Shuffle once on the host; each epoch visits contiguous minibatches in a
    # fresh random order (device views, no gather).
    perm0 = rng.permutation(thetas.shape[0])
    zt = ((targets[perm0] - self.shift) / self.scale).astype(np.float32)
    x_all = torch.from_numpy(np.ascontiguousarray(thetas[perm0], np.float32)).to(self.device)
    t_all = torch.from_numpy(np.ascontiguousarray(zt)).to(self.device)
    count = x_all.shape[0]
    nbatches = count // batch
    if nbatches < 1:
      raise ValueError(f"need at least one full batch of {batch} samples, got {count}")
    loss_buf = torch.zeros(1, dtype=torch.float64, device=self.device)
    epoch_loss = torch.zeros(1, dtype=torch.float64, device=self.device)
    dy = torch.empty((batch, self.out), dtype=torch.float32, device=self.device)
    dh2 = torch.empty((batch, self.hidden), dtype=torch.float32, device=self.device)
    dh1 = torch.empty_like(dh2)
    losses = []
    lib, st = self.lib, self._st()
    zero = self.zero_points() if hinge_weight > 0.0 else None
    total_steps, done = epochs * nbatches, 0
    for _ in range(epochs):
      epoch_loss.zero_()
      for bidx in rng.permutation(nbatches):
        s0 = int(bidx) * batch
        self.gradients(x_all[s0:s0 + batch], t_all[s0:s0 + batch], batch, dy, dh1, dh2,
                       loss_buf, hinge_weight, hinge_margin, zero)
        epoch_loss += loss_buf
        self.step += 1
        rate = lr * 0.5 * (1.0 + np.cos(np.pi * done / total_steps)) if cosine else lr
        done += 1
        for p, g, mm, vv in zip(self.params, self.grads, self.adam_m, self.adam_v):
          _lib.check(lib.qtqp_mlp_adam(p.data_ptr(), g.data_ptr(), mm.data_ptr(), vv.data_ptr(),
                                       p.numel(), float(rate), 0.9, 0.999, 1e-8, self.step, st))
      losses.append(float(epoch_loss.item()) / (nbatches * batch * self.out))
    self._wt16 = None  # the BF16 copies follow the new weights
    return TrainReport(epochs, losses[-1] if losses else float("nan"), losses)

  def predict_device(self, thetas: np.ndarray, threshold: float | None = None):
    """Warm-start tensors (x, y, active) laid out like the solver's x / y
    pools, for instances of the family in order; decoded on the device."""
    torch = self.torch
    count = thetas.shape[0]
    x = torch.from_numpy(np.ascontiguousarray(thetas, np.float32)).to(self.device)
    pred = self._forward_bf16(x, count) if self.bf16 else self._forward(x, count)[2]
    scale = torch.from_numpy(self.scale).to(self.device)
    shift = torch.from_numpy(self.shift).to(self.device)
    wx = torch.empty(count * self.n, dtype=torch.float64, device=self.device)
    wy = torch.empty(count * self.m, dtype=torch.float64, device=self.device)
    act = torch.empty(count * self.m, dtype=torch.uint8, device=self.device)
    thr = self.threshold if threshold is None else threshold
    _lib.check(self.lib.qtqp_mlp_decode(pred.data_ptr(), scale.data_ptr(), shift.data_ptr(),
                                        self.n, self.m, self.z, count, thr, wx.data_ptr(),
                                        wy.data_ptr(), act.data_ptr(), self._st()))
    return wx, wy, act

  def calibrate(self, thetas: np.ndarray, targets: np.ndarray, tight_cost: float = 2.0) -> float:
    """Picks the threshold on the predicted y_i - s_i that minimises the
    weighted count of misclassified inequality rows on (thetas, targets): a
    row wrongly held tight costs tight_cost, a row wrongly left free costs 1
    (a tight row that should be free needs more corrections of the reduced
    KKT solve to repair, so the threshold is biased up).  The truth is the
    sign of the target.  Sets self.threshold and self.row_error_rate (the
    plain fraction of misclassified rows at that threshold)."""
    n, z = self.n, self.z
    truth = targets[:, n + z:] > 0.0
    v = self.predict(thetas)[:, n + z:]
    spread = float(np.quantile(np.abs(v), 0.9)) if v.size else 1.0
    cands = np.concatenate([[0.0], spread * np.linspace(-0.5, 0.5, 41)])
    costs, errs = [], []
    for t in cands:
      pred = v > t
      false_tight = np.mean(pred & ~truth)
      false_free = np.mean(~pred & truth)
      costs.append(tight_cost * false_tight + false_free)
      errs.append(false_tight + false_free)
    best = int(np.argmin(costs))
    self.threshold = float(cands[best])
    self.row_error_rate = float(errs[best])
    return self.threshold

  def predict(self, thetas: np.ndarray) -> np.ndarray:
    """Unstandardised predictions [x; y_eq; y_ineq - s_ineq] on the host
    (count x (n + m))."""
    torch = self.torch
    x = torch.from_numpy(np.ascontiguousarray(thetas, np.float32)).to(self.device)
    count = thetas.shape[0]
    pred = self._forward_bf16(x, count) if self.bf16 else self._forward(x, count)[2]
    return pred.cpu().numpy().astype(np.float64) * self.scale + self.shift

  def params_host(self):
    return [p.cpu().numpy() for p in self.params]

  def save(self, path: str) -> None:
    """Weights, standardisation and threshold as an .npz file."""
    np.savez(path, *self.params_host(), scale=self.scale, shift=self.shift,
             threshold=self.threshold, dims=np.array([self.dim, self.n, self.m, self.z,
                                                      self.hidden]))

  @classmethod
  def load(cls, path: str, device=None) -> "WarmStartMLP":
    d = np.load(path)
    dim, n, m, z, hidden = (int(v) for v in d["dims"])
    net = cls(dim, n, m, z, hidden=hidden, device=device)
    for i, p in enumerate(net.params):
      p.copy_(net.torch.from_numpy(d[f"arr_{i}"]))
    net.scale, net.shift = d["scale"], d["shift"]
    net.threshold = float(d["threshold"])
    net._wt16 = None
    return net
