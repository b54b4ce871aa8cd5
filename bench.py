#!/usr/bin/env python
"""Benchmark: QPs solved per second on the batched uneven small-QP workload.

Workload (one "step"): 4096 independent dense QPs, n ~ U{8..64}, m = 2n,
z = n/4, A ~ N(0,1), P = L L^T + 1e-3 I (L n x n/2), b and c from a feasible
primal-dual pair; seeded (instance i of rank r: default_rng([1001, r*4096+i])).
All QPs are solved at atol=1e-7, rtol=1e-8 with every other QTQP.solve default,
in one persistent launch of the device-resident IPM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference ...   # the reference algorithm on host CPUs

Prints one JSON line (rank 0).  `value` is device-timed (inputs resident in
HBM, L2 flushed between steps); `e2e` adds the host->device copy of the
packed inputs and the device->host copy of x, y, s and statuses every step.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

METRIC = "QPs solved/s at atol 1e-7 (chosen form vs plain FP64, same B200); KKT TFLOP/s"
WORKLOAD = "batched uneven small dense QPs: 4096 x (n~U{8..64}, m=2n, z=n/4)"
COUNT = 4096
CPU_SAMPLE = 1024          # instances in the CPU-baseline sample
REF_SAMPLE = 1024          # instances per step of the reference arm
HBM_FALLBACK_GBS = 6650.0  # only if MEASURED_PEAKS.json is absent
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64 (non-tensor), nominal; for context only
# DRAM bytes (read + write) of one batch solve of this workload (all 8 group
# launches, the autotuned FP64 plan), from one ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum; None where no capture exists.
NCU_TRAFFIC_BYTES = {"fp64": 407.6e6, "mixed": None}


def _args():
  ap = argparse.ArgumentParser()
  ap.add_argument("--gpus", type=int, default=1)
  ap.add_argument("--steps", type=int, default=5)
  ap.add_argument("--warmup", type=int, default=3)
  ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
  ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64"],
                  help="form whose throughput is the headline value (both are measured)")
  ap.add_argument("--workload", default="batch_small",
                  choices=["batch_small", "dense_large", "mpc", "parametric", "sparse"],
                  help="batch_small: 4096 uneven small dense QPs (default); dense_large: "
                       "one n=4096, m=8192 dense QP on the whole GPU; parametric: a T=50 "
                       "MPC family with the learned warm start; sparse: one min-cost flow "
                       "QP on a grid network (supernodal factorisation)")
  ap.add_argument("--grid", type=int, default=60,
                  help="sparse: side of the grid network (n = 4 k (k - 1) edges)")
  ap.add_argument("--train", type=int, default=16384,
                  help="parametric: training instances (the family's stated split: 16384 "
                       "train, 3616 held out)")
  ap.add_argument("--warm-corrections", type=int, default=8,
                  help="parametric: primal-dual corrections of the reduced KKT solve")
  ap.add_argument("--warm-shift", type=float, default=0.1,
                  help="parametric: a rejected prediction starts the IPM shifted by this "
                       "(0: the cold start)")
  ap.add_argument("--hinge", type=float, default=1.0,
                  help="parametric: weight of the hinge term in the MLP training loss")
  ap.add_argument("--epochs", type=int, default=60, help="parametric: training epochs")
  ap.add_argument("--mpc-horizon", type=int, default=500,
                  help="mpc: horizon T (n = 60 T); 500 is the workload, smaller horizons are "
                       "for profiling captures")
  ap.add_argument("--mpc-parts", type=int, default=None,
                  help="mpc: partitions of the banded factorisation (default: the library's "
                       "choice for the band)")
  ap.add_argument("--large-n", type=int, default=4096,
                  help="dense_large: n (m = 2n, z = n/4); 4096 is the workload, smaller "
                       "sizes are for profiling captures")
  ap.add_argument("--count", type=int, default=COUNT)
  ap.add_argument("--no-cpu-baseline", action="store_true")
  ap.add_argument("--no-tune", action="store_true",
                  help="batch_small: use the library's default launch shapes")
  ap.add_argument("--tune-batch-pass", action="store_true",
                  help="batch_small: add the autotuner's pass over the whole concurrent batch")
  return ap.parse_args()


def _instances(rank: int, count: int, world: int = 1):
  """This rank's instances: all `count` at N = 1; at N > 1 its share of the
  world x count instances, balanced by estimated work (weak scaling: about
  `count` instances' work per GPU; only the rank's own instances are built)."""
  from qtqp_b200 import distributed, problems
  if world == 1:
    return [problems.small_dense_instance(i) for i in range(count)]
  total = world * count
  costs = [distributed.instance_cost(*problems.small_dense_size(i)) for i in range(total)]
  mine = distributed.shard_by_cost(costs, world)[rank]
  return [problems.small_dense_instance(i) for i in mine]


# ---------------------------------------------------------------------------
# CPU side: the oracle (a restatement of the reference algorithm) on host cores.
# ---------------------------------------------------------------------------
def _oracle_chunk(ids):
  os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
  from oracle import qtqp_oracle as orc
  from qtqp_b200 import problems
  solved = 0
  for i in ids:
    a, b, c, z, p = problems.small_dense_instance(i)
    if orc.solve(a, b, c, z, p, backend="dense").status == orc.STATUS_SOLVED:
      solved += 1
  return solved


def _cpu_pool(cores: int):
  """Spawned worker processes, one BLAS thread each (set before they start)."""
  os.environ["OPENBLAS_NUM_THREADS"] = "1"
  os.environ["OMP_NUM_THREADS"] = "1"
  return mp.get_context("spawn").Pool(cores)


def _time_oracle(pool, cores: int, ids) -> tuple[float, int]:
  chunks = [ids[k::cores] for k in range(cores)]
  t0 = time.perf_counter()
  solved = sum(pool.map(_oracle_chunk, chunks))
  return time.perf_counter() - t0, solved


def run_reference(args) -> None:
  rank = int(os.environ.get("RANK", "0"))
  if rank != 0:
    return
  cores = os.cpu_count() or 1
  with _cpu_pool(cores) as pool:
    _time_oracle(pool, cores, list(range(cores)))  # import warm-up
    for _ in range(args.warmup):
      _time_oracle(pool, cores, list(range(REF_SAMPLE)))
    times, solved = [], 0
    for _ in range(args.steps):
      ids = list(range(REF_SAMPLE))  # the first instances of the workload, every step
      t, s = _time_oracle(pool, cores, ids)
      times.append(t)
      solved += s
  total = sum(times)
  value = solved / total
  line = {
      "impl": "reference", "metric": METRIC, "value": value, "unit": "QPs/s",
      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
      "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
      "config": {"workload": WORKLOAD, "sample_per_step": REF_SAMPLE,
                 "backend": "dense Gram/Cholesky (SCIPY_DENSE algorithm)"},
      "cpu_baseline": {"value": value, "unit": "QPs/s", "cores": cores, "kind": "port",
                       "sample": f"the first {REF_SAMPLE} of the workload's {COUNT} instances "
                                 f"(generated and solved) every step, {args.steps} steps"},
      "e2e": {"value": value, "unit": "QPs/s", "h2d_bytes_per_step": 0,
              "d2h_bytes_per_step": 0},
  }
  print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side.
# ---------------------------------------------------------------------------
class _Clocks:
  """Samples nvidia-smi during the timed region."""

  Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
       "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
       "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

  def __init__(self, gpu_index: int):
    self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    self.proc = None
    try:
      self.proc = subprocess.Popen(
          ["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.Q}",
           "--format=csv,noheader,nounits", "-lms", "100"],
          stdout=self.f, stderr=subprocess.DEVNULL)
    except OSError:
      self.proc = None

  def stop(self) -> dict:
    if self.proc is None:
      return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    self.proc.terminate()
    self.proc.wait()
    self.f.seek(0)
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in self.f.read().splitlines():
      parts = [p.strip() for p in line.split(",")]
      if len(parts) < 9:
        continue
      try:
        sm.append(float(parts[1]))
        mx.append(float(parts[2]))
      except ValueError:
        continue
      for nm, val in zip(names, parts[5:9]):
        if val.lower() == "active":
          reasons.add(nm)
    os.unlink(self.f.name)
    return {"sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
            "samples": len(sm)}


def _peaks():
  path = os.path.join(ROOT, "MEASURED_PEAKS.json")
  if os.path.exists(path):
    with open(path) as f:
      d = json.load(f)
    return float(d["hbm_gbs"]), "measured"
  return HBM_FALLBACK_GBS, "fallback"


def run_ours(args) -> None:
  rank = int(os.environ.get("RANK", "0"))
  world = int(os.environ.get("WORLD_SIZE", "1"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  cpu = None
  # The oracle pool starts (spawn) before any CUDA call in this process.
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    cores = os.cpu_count() or 1
    with _cpu_pool(cores) as pool:
      _time_oracle(pool, cores, list(range(cores)))
      t, solved = _time_oracle(pool, cores, list(range(CPU_SAMPLE)))
    cpu = {"value": solved / t, "unit": "QPs/s", "cores": cores, "kind": "port",
           "sample": f"first {CPU_SAMPLE} of the {COUNT} instances, oracle restatement of "
                     f"the reference (dense Gram/Cholesky backend), one process per core"}

  import numpy as np
  import torch
  import qtqp_b200 as qb
  from qtqp_b200 import batch

  torch.cuda.set_device(local)
  dist = None
  if world > 1:
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
  dev = torch.device("cuda", local)
  stream = torch.cuda.current_stream(dev)

  insts = _instances(rank, args.count, world)
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in insts]

  # Launch shapes: the autotuner times each size class's candidate shapes on
  # this GPU (outside the timed region) unless --no-tune.
  from qtqp_b200 import autotune
  tuning, t_tune = None, 0.0
  if not args.no_tune:
    t0 = time.perf_counter()
    tuning = autotune.tune_dense_batch(qps, batch.SolveOptions(precision="fp64"), device=dev,
                                       batch_pass=args.tune_batch_pass)
    t_tune = time.perf_counter() - t0

  def prepare(precision):
    hb = batch.HostBatch(qps, batch.SolveOptions(precision=precision), pinned=True,
                         tuning=tuning)
    db = batch.DeviceBatch(hb, device=dev)
    db.upload(stream)
    torch.cuda.synchronize(dev)
    return hb, db

  flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

  def timed_kernel(db, steps, warmup):
    for _ in range(warmup):
      db.launch(stream)
    torch.cuda.synchronize(dev)
    total = 0.0
    for _ in range(steps):
      flush.fill_(1)
      e0 = torch.cuda.Event(enable_timing=True)
      e1 = torch.cuda.Event(enable_timing=True)
      e0.record(stream)
      db.launch(stream)
      e1.record(stream)
      e1.synchronize()
      total += e0.elapsed_time(e1) * 1e-3
    return total

  def barrier():
    if dist is not None:
      dist.barrier()
    torch.cuda.synchronize(dev)

  def max_over_ranks(v):
    if dist is None:
      return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())

  def sum_over_ranks(v):
    if dist is None:
      return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(round(t.item()))

  def solved_count(db):
    res, *_ = db.fetch()
    return int(np.sum(res["status"] == 0)), res

  # Plain FP64 form (comparator), then the chosen form.
  forms = {}
  for precision in ("fp64", "mixed"):
    hb, db = prepare(precision)
    barrier()
    clocks = _Clocks(local) if precision == args.precision else None
    t = timed_kernel(db, args.steps, args.warmup)
    ck = clocks.stop() if clocks else None
    barrier()
    t = max_over_ranks(t)
    solved, res = solved_count(db)
    forms[precision] = dict(hb=hb, db=db, time=t, solved=solved, res=res, clocks=ck)

  chosen = forms[args.precision]
  hb, db, res = chosen["hb"], chosen["db"], chosen["res"]
  solved_total = sum_over_ranks(chosen["solved"])
  value = solved_total * args.steps / chosen["time"]
  fp64_solved = sum_over_ranks(forms["fp64"]["solved"])
  mixed_solved = sum_over_ranks(forms["mixed"]["solved"])
  instances_total = sum_over_ranks(len(qps))
  fp64_value = fp64_solved * args.steps / forms["fp64"]["time"]
  same_status = bool(np.array_equal(forms["fp64"]["res"]["status"], res["status"]))

  def ev_pair():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

  # End to end through the public API: a list of CSC QTQP objects in, a list
  # of Solutions out (packing, planning, H2D copies, the solve, D2H copies,
  # unpacking), timed with CUDA events recorded before the call and after it
  # returns (the call synchronises).
  for _ in range(args.warmup):
    qb.solve_batch(qps, precision=args.precision, tuning=tuning)
  barrier()
  e_total, e2e_solved = 0.0, 0
  for _ in range(args.steps):
    flush.fill_(1)
    e0, e1 = ev_pair()
    e0.record(stream)
    sols = qb.solve_batch(qps, precision=args.precision, tuning=tuning)
    e1.record(stream)
    e1.synchronize()
    e_total += e0.elapsed_time(e1) * 1e-3
    e2e_solved = sum(1 for x in sols if x.status == qb.SolutionStatus.SOLVED)
  barrier()
  e_total = max_over_ranks(e_total)
  e2e_value = sum_over_ranks(e2e_solved) * args.steps / e_total
  h2d = hb.input_bytes
  d2h = db.output_bytes

  # The same through the C-ABI from already packed pinned pools (upload,
  # launch, download), and the two copies timed on their own.
  for _ in range(args.warmup):
    db.upload(stream)
    db.launch(stream)
    db.download(stream)
  barrier()
  d_total = h2d_t = d2h_t = 0.0
  for _ in range(args.steps):
    flush.fill_(1)
    e0, e1 = ev_pair()
    c0, c1 = ev_pair()
    c2, c3 = ev_pair()
    e0.record(stream)
    c0.record(stream)
    db.upload(stream)
    c1.record(stream)
    db.launch(stream)
    c2.record(stream)
    db.download(stream)
    c3.record(stream)
    e1.record(stream)
    e1.synchronize()
    d_total += e0.elapsed_time(e1) * 1e-3
    h2d_t += c0.elapsed_time(c1) * 1e-3
    d2h_t += c2.elapsed_time(c3) * 1e-3
  barrier()
  d_total = max_over_ranks(d_total)

  # Roofline of the dominant kernel (the batch kernel is the only one).
  iters = res["iterations"].astype(np.float64)
  ns = hb.inst["n"].astype(np.float64)
  ms = hb.inst["m"].astype(np.float64)
  bytes_per_iter = 8.0 * (ms * ns + ns * ns)          # A and P read once per IPM step
  alg_bytes = float(np.sum(iters * bytes_per_iter))
  factor_flops = float(np.sum((res["fp32_factorizations"] + res["fp64_factorizations"]) *
                              (ms * ns * (ns + 1) + ns ** 3 / 3.0)))
  t_launch = chosen["time"] / args.steps
  peak, peak_kind = _peaks()
  achieved = alg_bytes / t_launch / 1e9
  roofline = {
      "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
      "frac": achieved / peak, "peak_source": peak_kind,
      "traffic": NCU_TRAFFIC_BYTES.get(args.precision),
      "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum over one batch "
                         f"solve (8 launches), {args.precision} form, autotuned plan"
                         ) if NCU_TRAFFIC_BYTES.get(
                             args.precision) else "no capture of this form",
      "kernel": "dense_batch_kernel",
      "algorithmic_bytes_per_launch": alg_bytes,
      "kkt_factor_flops_per_launch": factor_flops,
      "kkt_tflops": factor_flops / t_launch / 1e12,
      "fp64_nominal_frac": factor_flops / t_launch / 1e12 / FP64_NOMINAL_TFLOPS,
  }
  if rank == 0:
    line = {
        "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * chosen["time"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distribution)",
        "config": {"workload": WORKLOAD, "instances_per_gpu": args.count,
                   "sharding": "one GPU" if world == 1 else
                               "cost-balanced shares of world x 4096 (m n^2 + n^3/3)",
                   "precision": args.precision, "l2": "flushed between steps (256 MiB write);"
                   " inputs also exceed L2",
                   "launch_groups": [list(g) for g in hb.groups],
                   "autotuned": None if tuning is None else {
                       "seconds": round(t_tune, 2),
                       "columns": ["n_lo", "n_hi", "block_threads", "lean", "onchip",
                                   "default_ms alone", "ms alone"],
                       "table": [[e["n_lo"], e["n_hi"], e["block_threads"], e["lean"],
                                  e["onchip"], e["default_ms"], e["ms"]] for e in tuning],
                       "batch_default_ms": tuning[0]["batch_default_ms"] if tuning else None,
                       "batch_ms": tuning[0]["batch_ms"] if tuning else None}},
        "fp64_value": fp64_value, "chosen_over_fp64": value / fp64_value,
        "mixed_value": mixed_solved * args.steps / forms["mixed"]["time"],
        "mixed_statuses_identical_to_fp64": bool(np.array_equal(
            forms["fp64"]["res"]["status"], forms["mixed"]["res"]["status"])),
        "statuses_identical_to_fp64": same_status,
        "solved_per_step": solved_total, "instances_per_step": instances_total,
        "mean_iterations": float(np.mean(iters)),
        "factorizations": {"fp32": int(res["fp32_factorizations"].sum()),
                           "fp64": int(res["fp64_factorizations"].sum())},
        "e2e": {"value": e2e_value, "unit": "QPs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "qtqp.solve_batch(list of CSC QTQP) -> list of Solution",
                "ms_per_step": 1e3 * e_total / args.steps},
        "e2e_device_api": {"value": solved_total * args.steps / d_total, "unit": "QPs/s",
                           "path": "C-ABI from packed pinned pools: H2D, solve, D2H",
                           "ms_per_step": 1e3 * d_total / args.steps,
                           "h2d_ms": 1e3 * h2d_t / args.steps,
                           "d2h_ms": 1e3 * d2h_t / args.steps},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": chosen["clocks"],
        "gpu_launches": args.steps * int(hb.plan.num_groups),
    }
    print(json.dumps(line), flush=True)
  if dist is not None:
    dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Other workloads (not the default line): one large dense QP, and the
# parametric MPC family with the learned warm start.
# ---------------------------------------------------------------------------
LARGE_WORKLOAD = "one large dense QP: n=4096, m=8192, z=1024 (A ~ N(0,1/n), P = U diag(d) U^T + 1e-4 I)"
PARAM_WORKLOAD = "parametric MPC family T=50 (n=3000, m=8000, z=2000): (b, c) = (b0, c0) + W theta"


_PARAM_FAMILY = {}


def _param_oracle_chunk(spec):
  """Solves instances `ids` of the parametric family (built once per worker
  process) with the oracle's sparse-LU backend; returns how many it solved."""
  os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
  from oracle import qtqp_oracle as orc
  from qtqp_b200 import problems
  count, ids = spec
  if count not in _PARAM_FAMILY:
    _PARAM_FAMILY[count] = problems.parametric_mpc_family(count=count)
  fam = _PARAM_FAMILY[count]
  for i in ids:
    a, b, c, z, p = problems.parametric_mpc_instance(fam, i)
    orc.solve(a, b, c, z, p, backend="superlu")
  return len(ids)


def _bf16_peak():
  path = os.path.join(ROOT, "MEASURED_PEAKS.json")
  if os.path.exists(path):
    with open(path) as f:
      return float(json.load(f)["bf16_tflops"]), "measured"
  return 1590.0, "fallback"


def _ev_time(stream, fn):
  import torch
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record(stream)
  fn()
  e1.record(stream)
  e1.synchronize()
  return e0.elapsed_time(e1) * 1e-3


def run_dense_large(args):
  """One large dense QP per step on the whole GPU (replicas only for N > 1)."""
  rank = int(os.environ.get("RANK", "0"))
  world = int(os.environ.get("WORLD_SIZE", "1"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  from qtqp_b200 import problems
  nl = args.large_n
  a, b, c, z, p = problems.large_dense(seed=1002 + rank, n=nl, m=2 * nl, z=nl // 4,
                                   rank=min(256, nl // 4))
  m, n = a.shape
  flops = m * n * (n + 1) + n ** 3 / 3.0  # one factorisation (Gram + Cholesky)
  if args.impl == "reference":
    if rank != 0:
      return
    import scipy.sparse as sp
    from oracle import qtqp_oracle as orc
    times = []
    for step in range(args.warmup + args.steps):
      t0 = time.perf_counter()
      r = orc.solve(sp.csc_matrix(a), b, c, z, sp.csc_matrix(p), backend="dense")
      if step >= args.warmup:
        times.append(time.perf_counter() - t0)
    value = len(times) / sum(times)
    cores = os.cpu_count() or 1
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": LARGE_WORKLOAD, "status": r.status},
        "cpu_baseline": {"value": value, "unit": "QPs/s", "cores": cores, "kind": "port",
                         "sample": "the whole QP, oracle restatement (dense Gram/Cholesky, "
                                   "multithreaded BLAS)"},
        "e2e": {"value": value, "unit": "QPs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)
    return
  cpu = None
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    import scipy.sparse as sp
    from oracle import qtqp_oracle as orc
    t0 = time.perf_counter()
    orc.solve(sp.csc_matrix(a), b, c, z, sp.csc_matrix(p), backend="dense")
    t = time.perf_counter() - t0
    cpu = {"value": 1.0 / t, "unit": "QPs/s", "cores": os.cpu_count() or 1, "kind": "port",
           "sample": "one whole solve of the QP, oracle restatement (dense Gram/Cholesky, "
                     "multithreaded BLAS)"}
  import numpy as np
  import torch
  from qtqp_b200 import batch, large
  torch.cuda.set_device(local)
  dev = torch.device("cuda", local)
  stream = torch.cuda.current_stream(dev)
  dist = None
  if world > 1:
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
  prob = batch.DenseProblem(a=a, b=b, c=c, z=z, p=p)
  forms = {}
  for precision in ("fp64", "mixed"):
    dl = large.DeviceLarge(prob, batch.SolveOptions(precision=precision), device=dev)
    dl.upload(stream)
    for _ in range(args.warmup):
      dl.launch(stream)
    torch.cuda.synchronize(dev)
    clocks = _Clocks(local) if precision == args.precision else None
    t = sum(_ev_time(stream, lambda: dl.launch(stream)) for _ in range(args.steps))
    ck = clocks.stop() if clocks else None
    res = dl.fetch()[0][0]
    if dist is not None:
      tt = torch.tensor([t], dtype=torch.float64, device=dev)
      dist.all_reduce(tt, op=dist.ReduceOp.MAX)
      t = float(tt.item())
    forms[precision] = dict(dl=dl, time=t, res=res, clocks=ck)
  chosen = forms[args.precision]
  dl, res = chosen["dl"], chosen["res"]
  solved = int(res["status"] == 0)
  value = solved * world * args.steps / chosen["time"]
  fp64 = forms["fp64"]
  fp64_value = int(fp64["res"]["status"] == 0) * world * args.steps / fp64["time"]
  mixed = forms["mixed"]
  mixed_value = int(mixed["res"]["status"] == 0) * world * args.steps / mixed["time"]
  # End to end: host inputs -> device, solve, outputs -> host, every step.
  h_out = [torch.empty_like(t_, device="cpu").pin_memory() for t_ in (dl.x, dl.y, dl.s,
                                                                      dl.result)]

  def e2e_step():
    dl.upload(stream)
    dl.launch(stream)
    with torch.cuda.stream(stream):
      for dst, src in zip(h_out, (dl.x, dl.y, dl.s, dl.result)):
        dst.copy_(src, non_blocking=True)
  e2e_step()
  e_total = sum(_ev_time(stream, e2e_step) for _ in range(args.steps))
  t_launch = chosen["time"] / args.steps
  nfact = int(res["fp32_factorizations"] + res["fp64_factorizations"])
  achieved = flops * nfact / t_launch / 1e12
  peak, peak_kind = _bf16_peak()
  if rank == 0:
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_launch,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distribution)",
        "config": {"workload": LARGE_WORKLOAD if nl == 4096 else
                   f"one dense QP: n={nl}, m={2 * nl}, z={nl // 4} (profiling size)",
                   "precision": args.precision,
                   "l2": "inputs (A 268 MB, P 134 MB) exceed L2",
                   "parallelism": "replicas" if world > 1 else "one QP per GPU"},
        "fp64_value": fp64_value, "mixed_value": mixed_value,
        "chosen_over_fp64": value / fp64_value if fp64_value else None,
        "statuses_identical": bool(fp64["res"]["status"] == mixed["res"]["status"]),
        "iterations": int(res["iterations"]),
        "factorizations": {"fp32": int(res["fp32_factorizations"]),
                           "fp64": int(res["fp64_factorizations"])},
        "kkt_tflops": achieved,
        "e2e": {"value": solved * args.steps / e_total, "unit": "QPs/s",
                "h2d_bytes_per_step": dl.input_bytes,
                "d2h_bytes_per_step": sum(int(t_.numel() * t_.element_size()) for t_ in h_out)},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                     "kernel": "large_solve_kernel",
                     "algorithmic_flops_per_launch": flops * nfact,
                     "note": "algorithmic KKT factorisation flops (m n (n+1) + n^3/3 per "
                             "factorisation) over the whole solve's time"},
        "cpu_baseline": cpu, "clocks": chosen["clocks"], "gpu_launches": args.steps}),
          flush=True)
  if dist is not None:
    dist.destroy_process_group()


MPC_WORKLOAD = ("one MPC-structured QP: horizon T, nx=40, nu=20 (n=60T, z=40T, m=z+2n), "
                "box bounds 5 / 1, 10% of the boxes active")


def run_mpc(args):
  """One banded MPC QP per step (replicas only for N > 1)."""
  rank = int(os.environ.get("RANK", "0"))
  world = int(os.environ.get("WORLD_SIZE", "1"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  from qtqp_b200 import problems
  T = args.mpc_horizon
  a, b, c, z, p = problems.mpc_feasible(T)
  workload = MPC_WORKLOAD.replace("horizon T", f"horizon T={T}")
  if args.impl == "reference":
    # Rank 0 alone: one whole oracle solve per step (SuperLU factorises on one
    # thread; the problem is a single QP).
    if rank != 0:
      return
    from oracle import qtqp_oracle as orc
    times = []
    for step in range(args.warmup + args.steps):
      t0 = time.perf_counter()
      r = orc.solve(a, b, c, z, p, backend="superlu")
      if step >= args.warmup:
        times.append(time.perf_counter() - t0)
    t_cpu = sum(times) / len(times)
    cpu = {"value": 1.0 / t_cpu, "unit": "QPs/s", "cores": 1, "kind": "port",
           "sample": f"one whole solve per step, {args.steps} steps, oracle restatement "
                     "(SuperLU KKT)"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": 1.0 / t_cpu, "unit": "QPs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_cpu, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "status": r.status}, "cpu_baseline": cpu,
        "e2e": {"value": 1.0 / t_cpu, "unit": "QPs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)
    return
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    from oracle import qtqp_oracle as orc
    t0 = time.perf_counter()
    orc.solve(a, b, c, z, p, backend="superlu")
    t_cpu = time.perf_counter() - t0
    cpu = {"value": 1.0 / t_cpu, "unit": "QPs/s", "cores": 1, "kind": "port",
           "sample": "one whole solve, oracle restatement (SuperLU KKT)"}
  else:
    cpu = None
  import numpy as np
  import torch
  import qtqp_b200 as qb
  from qtqp_b200 import band, batch
  torch.cuda.set_device(local)
  dev = torch.device("cuda", local)
  stream = torch.cuda.current_stream(dev)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  forms = {}
  for precision in ("fp64", "mixed"):
    hb = band.HostBandBatch([q.band_problem()], batch.SolveOptions(precision=precision))
    db = band.DeviceBandGrid(hb, device=dev, parts=args.mpc_parts)
    db.upload(stream)
    for _ in range(args.warmup):
      db.launch(stream)
    torch.cuda.synchronize(dev)
    clocks = _Clocks(local) if precision == args.precision else None
    t = sum(_ev_time(stream, lambda: db.launch(stream)) for _ in range(args.steps))
    ck = clocks.stop() if clocks else None
    forms[precision] = dict(hb=hb, db=db, time=t, res=db.fetch()[0][0], clocks=ck)
  chosen = forms[args.precision]
  hb, db, res = chosen["hb"], chosen["db"], chosen["res"]
  value = int(res["status"] == 0) * args.steps / chosen["time"]
  fp64 = forms["fp64"]
  mixed = forms["mixed"]
  h_out = [torch.empty_like(t_, device="cpu").pin_memory() for t_ in (db.x, db.y, db.s)]

  def e2e_step():
    db.upload(stream)
    db.launch(stream)
    with torch.cuda.stream(stream):
      for dst, src in zip(h_out, (db.x, db.y, db.s)):
        dst.copy_(src, non_blocking=True)
  e2e_step()
  e_total = sum(_ev_time(stream, e2e_step) for _ in range(args.steps))
  t_launch = chosen["time"] / args.steps
  nnz = int(hb.inst["nnz_a"][0])
  n_, m_ = int(hb.inst["n"][0]), int(hb.inst["m"][0])
  iters = int(res["iterations"])
  # Algorithmic bytes per IPM iteration: the SpMV bytes of A x in CSR (
  # 12 nnz + 4 (rows + 1) + 8 (cols + rows)), twice (A x and A^T y), plus the
  # band factor written and read (8 n (bw + 1) each).
  bw = int(hb.inst["bw"][0])
  per_iter = 2 * (12 * nnz + 4 * (m_ + 1) + 8 * (n_ + m_)) + 2 * 8 * n_ * (bw + 1)
  achieved = per_iter * iters / t_launch / 1e9
  peak, peak_kind = _peaks()
  if rank == 0:
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_launch, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distribution)",
        "config": {"workload": workload, "precision": args.precision, "bandwidth": bw,
                   "partitions": db.parts,
                   "parallelism": "replicas" if world > 1 else "one QP per GPU"},
        "fp64_value": int(fp64["res"]["status"] == 0) * args.steps / fp64["time"],
        "mixed_value": int(mixed["res"]["status"] == 0) * args.steps / mixed["time"],
        "statuses_identical": bool(fp64["res"]["status"] == mixed["res"]["status"]),
        "iterations": iters,
        "factorizations": {"fp32": int(res["fp32_factorizations"]),
                           "fp64": int(res["fp64_factorizations"])},
        "e2e": {"value": int(res["status"] == 0) * args.steps / e_total, "unit": "QPs/s",
                "h2d_bytes_per_step": hb.input_bytes,
                "d2h_bytes_per_step": sum(int(t_.numel() * t_.element_size()) for t_ in h_out)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                     "kernel": "band_grid_kernel",
                     "algorithmic_bytes_per_launch": per_iter * iters},
        "cpu_baseline": cpu, "clocks": chosen["clocks"], "gpu_launches": args.steps}),
          flush=True)


SPARSE_WORKLOAD = ("one min-cost flow QP on a k x k grid network (both directions of every "
                   "edge, quadratic costs): n = 4 k (k - 1), node conservation equalities, "
                   "0 <= x <= u")


def run_sparse(args):
  """One sparse QP per step on the supernodal whole-GPU path (replicas only
  for N > 1)."""
  rank = int(os.environ.get("RANK", "0"))
  world = int(os.environ.get("WORLD_SIZE", "1"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  from qtqp_b200 import problems
  k = args.grid
  a, b, c, z, p = problems.grid_flow(k)
  workload = SPARSE_WORKLOAD.replace("k x k", f"{k} x {k}")
  if args.impl == "reference":
    if rank != 0:
      return
    from oracle import qtqp_oracle as orc
    times = []
    for step in range(args.warmup + args.steps):
      t0 = time.perf_counter()
      r = orc.solve(a, b, c, z, p, backend="superlu")
      if step >= args.warmup:
        times.append(time.perf_counter() - t0)
    t_cpu = sum(times) / len(times)
    cpu = {"value": 1.0 / t_cpu, "unit": "QPs/s", "cores": 1, "kind": "port",
           "sample": f"one whole solve per step, {args.steps} steps, oracle restatement "
                     "(SuperLU KKT)"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": 1.0 / t_cpu, "unit": "QPs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_cpu, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "status": r.status}, "cpu_baseline": cpu,
        "e2e": {"value": 1.0 / t_cpu, "unit": "QPs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)
    return
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    from oracle import qtqp_oracle as orc
    t0 = time.perf_counter()
    orc.solve(a, b, c, z, p, backend="superlu")
    t_cpu = time.perf_counter() - t0
    cpu = {"value": 1.0 / t_cpu, "unit": "QPs/s", "cores": 1, "kind": "port",
           "sample": "one whole solve, oracle restatement (SuperLU KKT)"}
  else:
    cpu = None
  import torch
  import qtqp_b200 as qb
  from qtqp_b200 import batch, sparse
  torch.cuda.set_device(local)
  dev = torch.device("cuda", local)
  stream = torch.cuda.current_stream(dev)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  t0 = time.perf_counter()
  plan = q.sparse_plan()
  t_plan = time.perf_counter() - t0
  prob = plan.permuted(q.a, q.b, q.c, q.z, q.p if q.p.nnz else None)
  forms = {}
  for precision in ("fp64", "mixed"):
    dg = sparse.DeviceSparseGrid(prob, plan, batch.SolveOptions(precision=precision), device=dev)
    dg.upload(stream)
    for _ in range(args.warmup):
      dg.launch(stream)
    torch.cuda.synchronize(dev)
    clocks = _Clocks(local) if precision == args.precision else None
    t = sum(_ev_time(stream, lambda: dg.launch(stream)) for _ in range(args.steps))
    ck = clocks.stop() if clocks else None
    forms[precision] = dict(dg=dg, time=t, res=dg.fetch()[0][0], clocks=ck)
  chosen = forms[args.precision]
  dg, res = chosen["dg"], chosen["res"]
  value = int(res["status"] == 0) * args.steps / chosen["time"]
  fp64, mixed = forms["fp64"], forms["mixed"]
  # End to end through the public API: solve_batch on the QTQP (its symbolic
  # plan is cached on it after the first call), host packing, copies, solve,
  # read-back and the Solution, timed with CUDA events.
  qb.solve_batch([q], storage="sparse", precision=args.precision)
  e_total = sum(_ev_time(stream, lambda: qb.solve_batch([q], storage="sparse",
                                                        precision=args.precision))
                for _ in range(args.steps))
  t_launch = chosen["time"] / args.steps
  d = plan.desc
  iters = int(res["iterations"])
  nnz = int(dg.pools.inst["nnz_a"][0])
  n_, m_ = int(dg.pools.inst["n"][0]), int(dg.pools.inst["m"][0])
  # Algorithmic bytes per IPM iteration: the SpMV bytes of A x in CSR (12 nnz
  # + 4 (rows + 1) + 8 (cols + rows)), twice (A x and A^T y), plus the
  # supernodal factor written and read (8 bytes per stored value each).
  per_iter = 2 * (12 * nnz + 4 * (m_ + 1) + 8 * (n_ + m_)) + 2 * 8 * int(d.nvals)
  achieved = per_iter * iters / t_launch / 1e9
  peak, peak_kind = _peaks()
  nfact = int(res["fp32_factorizations"] + res["fp64_factorizations"])
  if rank == 0:
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_launch, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distribution)",
        "config": {"workload": workload, "n": n_, "m": m_, "precision": args.precision,
                   "supernodes": int(d.nsuper), "top_levels": int(d.top_levels),
                   "nnz_l": int(d.nnz_l), "fill_of_dense": plan.fill_fraction(),
                   "symbolic_seconds": t_plan,
                   "parallelism": "replicas" if world > 1 else "one QP per GPU"},
        "fp64_value": int(fp64["res"]["status"] == 0) * args.steps / fp64["time"],
        "mixed_value": int(mixed["res"]["status"] == 0) * args.steps / mixed["time"],
        "statuses_identical": bool(fp64["res"]["status"] == mixed["res"]["status"]),
        "iterations": iters,
        "factorizations": {"fp32": int(res["fp32_factorizations"]),
                           "fp64": int(res["fp64_factorizations"])},
        "kkt_tflops": d.flops * nfact / t_launch / 1e12,
        "e2e": {"value": int(res["status"] == 0) * args.steps / e_total, "unit": "QPs/s",
                "h2d_bytes_per_step": dg.input_bytes,
                "d2h_bytes_per_step": 8 * (n_ + 2 * m_) + _lib_result_bytes(),
                "path": "qtqp.solve_batch([QTQP], storage='sparse') -> [Solution]"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                     "kernel": "sparse_grid_kernel",
                     "algorithmic_bytes_per_launch": per_iter * iters},
        "cpu_baseline": cpu, "clocks": chosen["clocks"], "gpu_launches": args.steps}),
          flush=True)


def _lib_result_bytes() -> int:
  from qtqp_b200 import _lib
  return int(_lib.RESULT_DTYPE.itemsize)


def run_parametric(args):
  """Plain FP64 batch vs mixed precision + learned warm start on held-out
  instances of the parametric family (training is outside the timed region)."""
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  if rank != 0:
    return
  test_count = args.count if args.count != COUNT else 3616
  from qtqp_b200 import problems
  fam = problems.parametric_mpc_family(count=args.train + test_count)
  thetas = fam[-1]
  insts = [problems.parametric_mpc_instance(fam, i) for i in range(args.train + test_count)]
  if args.impl == "reference":
    # One held-out instance per host core per step, each core a spawned
    # process with one BLAS thread; instances cycle through the held-out set.
    cores = os.cpu_count() or 1
    total = args.train + test_count
    held_out = list(range(args.train, total))
    times, done, nxt = [], 0, 0
    with _cpu_pool(cores) as pool:
      for step in range(args.warmup + args.steps):
        ids = [held_out[(nxt + k) % len(held_out)] for k in range(cores)]
        nxt += cores
        t0 = time.perf_counter()
        solved = sum(pool.map(_param_oracle_chunk, [(total, [i]) for i in ids]))
        if step >= args.warmup:
          times.append(time.perf_counter() - t0)
          done += solved
    t = sum(times)
    value = done / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": PARAM_WORKLOAD},
        "cpu_baseline": {"value": value, "unit": "QPs/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} held-out instances per step (one per core), "
                                   f"{args.steps} steps, oracle (sparse LU)"},
        "e2e": {"value": value, "unit": "QPs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)
    return
  import numpy as np
  import torch
  import qtqp_b200 as qb
  from qtqp_b200 import band, batch, warmstart
  torch.cuda.set_device(local)
  dev = torch.device("cuda", local)
  stream = torch.cuda.current_stream(dev)
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in insts]
  train = list(range(args.train))
  test = list(range(args.train, args.train + test_count))
  t0 = time.perf_counter()
  sols = qb.solve_batch([qps[i] for i in train], storage="band")
  t_label = time.perf_counter() - t0
  keep = [i for i, s_ in zip(train, sols) if s_.status == qb.SolutionStatus.SOLVED]
  sols = [s_ for s_ in sols if s_.status == qb.SolutionStatus.SOLVED]
  q0 = qps[0]
  targets = warmstart.targets_from(q0.n, q0.z, [s_.x for s_ in sols], [s_.y for s_ in sols],
                                   [s_.s for s_ in sols])
  net = warmstart.WarmStartMLP(dim=thetas.shape[1], n=q0.n, m=q0.m, z=q0.z, seed=0, device=dev)
  t0 = time.perf_counter()
  rep = net.train(thetas[keep], targets, epochs=args.epochs, batch=64, lr=2e-3,
                  hinge_weight=args.hinge, cosine=True)
  torch.cuda.synchronize(dev)
  t_train = time.perf_counter() - t0
  net.calibrate(thetas[keep], targets)
  probs = [qps[i].band_problem() for i in test]

  def timed(opts, warm_fn):
    hb = band.HostBandBatch(probs, opts)
    db = band.DeviceBandBatch(hb, device=dev)
    db.upload(stream)
    for _ in range(args.warmup):
      db.launch(stream, warm=warm_fn())
    torch.cuda.synchronize(dev)
    t = sum(_ev_time(stream, lambda: db.launch(stream, warm=warm_fn()))
            for _ in range(args.steps))
    return t, db.fetch()[0]
  t_plain, r_plain = timed(batch.SolveOptions(precision="fp64"), lambda: None)
  corr = args.warm_corrections
  t_warm, r_warm = timed(batch.SolveOptions(precision=args.precision, warm_corrections=corr,
                                            warm_shift=args.warm_shift),
                         lambda: net.predict_device(thetas[test]))
  solved_w = int(np.sum(r_warm["status"] == 0))
  solved_p = int(np.sum(r_plain["status"] == 0))
  value = solved_w * args.steps / t_warm
  fp64_value = solved_p * args.steps / t_plain
  hidden = net.hidden
  params = thetas.shape[1] * hidden + hidden * hidden + hidden * net.out + 2 * hidden + net.out
  train_flops = 3 * 2 * params * len(keep) * rep.epochs
  print(json.dumps({
      "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": 1, "steps": args.steps,
      "warmup": args.warmup, "ms_per_step": 1e3 * t_warm / args.steps, "higher_is_better": True,
      "scaling": "weak", "vs_baseline": None, "dtype": "f64",
      "data": "synthetic (seeded generator of the family)",
      "config": {"workload": PARAM_WORKLOAD, "test_instances": test_count,
                 "train_instances": len(keep), "warm_corrections": corr,
                 "warm_shift": args.warm_shift, "hinge_weight": args.hinge,
                 "epochs": rep.epochs,
                 "chosen": f"{args.precision} + learned warm start; fp64_value: plain FP64"},
      "fp64_value": fp64_value, "chosen_over_fp64": value / fp64_value,
      "statuses_identical": bool(np.array_equal(r_plain["status"], r_warm["status"])),
      "warm_accepted": int(r_warm["warm_started"].sum()),
      "iterations": {"plain": int(r_plain["iterations"].sum()),
                     "warm": int(r_warm["iterations"].sum())},
      "mlp": {"train_seconds": t_train, "label_seconds": t_label, "epochs": rep.epochs,
              "final_loss": rep.final_loss, "row_error_rate": net.row_error_rate,
              "train_tflops": train_flops / t_train / 1e12},
      "cpu_baseline": None, "gpu_launches": args.steps * 5}), flush=True)


def main():
  args = _args()
  if args.workload == "dense_large":
    run_dense_large(args)
  elif args.workload == "parametric":
    run_parametric(args)
  elif args.workload == "sparse":
    run_sparse(args)
  elif args.workload == "mpc":
    run_mpc(args)
  elif args.impl == "reference":
    run_reference(args)
  else:
    run_ours(args)


if __name__ == "__main__":
  main()
