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
# DRAM bytes (read + write) of one batch solve (its 8 group launches, mixed
# precision) on this workload, from an ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum (profiles/dense_batch_kernel_config1.md).
NCU_TRAFFIC_BYTES = 171.6e6


def _args():
  ap = argparse.ArgumentParser()
  ap.add_argument("--gpus", type=int, default=1)
  ap.add_argument("--steps", type=int, default=5)
  ap.add_argument("--warmup", type=int, default=3)
  ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
  ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
  ap.add_argument("--count", type=int, default=COUNT)
  ap.add_argument("--no-cpu-baseline", action="store_true")
  return ap.parse_args()


def _instances(rank: int, count: int):
  from qtqp_b200 import problems
  return [problems.config1_instance(rank * COUNT + i) for i in range(count)]


# ---------------------------------------------------------------------------
# CPU side: the oracle (a restatement of the reference algorithm) on host cores.
# ---------------------------------------------------------------------------
def _oracle_chunk(ids):
  os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
  from oracle import qtqp_oracle as orc
  from qtqp_b200 import problems
  solved = 0
  for i in ids:
    a, b, c, z, p = problems.config1_instance(i)
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
    for k in range(args.steps):
      ids = list(range(k * REF_SAMPLE, (k + 1) * REF_SAMPLE))
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
                       "sample": f"{REF_SAMPLE} instances per step, {args.steps} steps"},
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

  insts = _instances(rank, args.count)
  qps = [qb.QTQP(a=a, b=b, c=c, z=z, p=p) for a, b, c, z, p in insts]
  probs = [q.dense_problem() for q in qps]

  def prepare(precision):
    hb = batch.HostBatch(probs, batch.SolveOptions(precision=precision))
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

  def solved_count(db):
    res, *_ = db.fetch()
    return int(np.sum(res["status"] == 0)), res

  # Plain FP64 form (comparator), then the chosen form.
  forms = {}
  for precision in ("fp64", args.precision) if args.precision != "fp64" else ("fp64",):
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
  solved_total = chosen["solved"] * world
  value = solved_total * args.steps / chosen["time"]
  fp64_value = forms["fp64"]["solved"] * world * args.steps / forms["fp64"]["time"]
  same_status = bool(np.array_equal(forms["fp64"]["res"]["status"], res["status"]))

  # End to end through the C-ABI with host buffers: H2D inputs, solve, D2H outputs.
  h_out = [torch.empty_like(t, device="cpu").pin_memory() for t in (db.x, db.y, db.s,
                                                                   db.results)]
  for _ in range(args.warmup):
    db.upload(stream)
    db.launch(stream)
  barrier()
  e_total = 0.0
  for _ in range(args.steps):
    flush.fill_(1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    db.upload(stream)
    db.launch(stream)
    with torch.cuda.stream(stream):
      for dst, src in zip(h_out, (db.x, db.y, db.s, db.results)):
        dst.copy_(src, non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    e_total += e0.elapsed_time(e1) * 1e-3
  barrier()
  e_total = max_over_ranks(e_total)
  e2e_value = solved_total * args.steps / e_total
  h2d = hb.input_bytes
  d2h = sum(int(t.numel() * t.element_size()) for t in h_out)

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
      "traffic": NCU_TRAFFIC_BYTES,
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
                   "precision": args.precision, "l2": "flushed between steps (256 MiB write);"
                   " inputs also exceed L2",
                   "launch_groups": [list(g) for g in hb.groups]},
        "fp64_value": fp64_value, "chosen_over_fp64": value / fp64_value,
        "statuses_identical_to_fp64": same_status,
        "solved_per_step": solved_total, "instances_per_step": args.count * world,
        "mean_iterations": float(np.mean(iters)),
        "factorizations": {"fp32": int(res["fp32_factorizations"].sum()),
                           "fp64": int(res["fp64_factorizations"].sum())},
        "e2e": {"value": e2e_value, "unit": "QPs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": chosen["clocks"],
        "gpu_launches": args.steps * int(hb.plan.num_groups),
    }
    print(json.dumps(line), flush=True)
  if dist is not None:
    dist.destroy_process_group()


def main():
  args = _args()
  if args.impl == "reference":
    run_reference(args)
  else:
    run_ours(args)


if __name__ == "__main__":
  main()
