"""Autotuner of the dense batch's launch shapes (no reference counterpart).

The batch solve runs one persistent launch per size class of the instances
(qtqp_dense_batch_plan); how fast a class solves depends on its launch
shape: threads per block, the register-capped ("lean") or unrestricted
kernel, and whether A and P stay in shared memory or are read through L2.
The default plan chooses by heuristics.  tune_dense_batch times every
candidate shape on each launch group of a representative batch, on the
device (CUDA events), in one or two stages:

1. each group launched alone, keeping its fastest shape;
2. (optional) the whole batch, whose groups run concurrently on side
   streams, timed as a caller sees it (L2 flushed before each solve): one pass
   of coordinate descent over the groups (largest first) that changes a
   group's shape only when the whole solve gets faster.  A group that is
   fastest alone with large blocks (low latency per QP) can be faster inside
   the batch with small ones (more QPs per SM), because the other groups
   fill the GPU meanwhile.

It returns a table of {n_lo, n_hi, block_threads, lean, onchip} entries that
qtqp_dense_batch_plan_tuned applies to later plans.  Tables are cached per
GPU model in a JSON file (save / load), which solve_batch picks up.
"""

from __future__ import annotations

import json
import os

import numpy as np

from . import _lib
from . import batch as _batch

CANDIDATES = [(nt, lean, onchip) for nt in (64, 128, 256) for lean in (0, 1)
              for onchip in (0, 1)]
# Single-warp blocks (barriers become warp syncs) are tried for the classes of
# small QPs only, where one warp has enough work.
SMALL_N = 32
SMALL_CANDIDATES = [(32, lean, onchip) for lean in (0, 1) for onchip in (0, 1)]


def cache_path() -> str:
  """The tuning cache: $QTQP_TUNING_FILE, else ~/.cache/qtqp_b200/tuning.json."""
  return os.environ.get("QTQP_TUNING_FILE") or os.path.join(
      os.path.expanduser("~"), ".cache", "qtqp_b200", "tuning.json")


def _gpu_key(torch, device) -> str:
  return torch.cuda.get_device_name(device)


def _time_group(torch, db, g, stream, reps) -> float:
  db.launch_group(g, stream)  # warm-up
  best = float("inf")
  for _ in range(reps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    db.launch_group(g, stream)
    e1.record(stream)
    e1.synchronize()
    best = min(best, e0.elapsed_time(e1))
  return best


def _time_batch(torch, db, stream, reps, flush) -> float:
  """Mean ms of `reps` whole-batch solves, each after a write of `flush` (a
  buffer larger than L2), as a caller that solves one batch at a time sees
  them."""
  db.launch(stream)  # warm-up
  total = 0.0
  for _ in range(reps):
    flush.fill_(1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    db.launch(stream)
    e1.record(stream)
    e1.synchronize()
    total += e0.elapsed_time(e1)
  return total / reps


def tune_dense_batch(problems, opts: _batch.SolveOptions | None = None, candidates=None,
                     reps: int = 3, device=None, batch_pass: bool = False) -> list[dict]:
  """Times each candidate (block_threads, lean, onchip) on every launch group
  of the default plan of `problems` and returns the tuning table of the
  chosen shapes.  Each entry carries ms and default_ms (the group launched
  alone with the chosen and the default shape) and batch_ms and
  batch_default_ms (the whole batch solve with the table and with the
  default plan).  A candidate that changes any instance's status against the
  default shape is never chosen.  batch_pass=True adds the second stage (on
  the 4096 small dense QPs it measured no gain over the first stage alone:
  160.0k / 157.7k against 160.0k / 157.2k QPs/s in two bench runs each, for
  12 s more tuning, so it is off by default)."""
  torch = _lib.require_device()
  opts = opts or _batch.SolveOptions()
  dev = torch.device(device or "cuda")
  stream = torch.cuda.current_stream(dev)
  hb = _batch.HostBatch(problems, opts, pinned=True)
  db = _batch.DeviceBatch(hb, device=dev, records=False)
  db.upload(stream)
  groups = [(hb.group_n_range(g), hb.plan.groups[g]) for g in range(hb.plan.num_groups)]
  alone = {}    # (group, candidate) -> ms alone (valid candidates only)
  default = {}  # group -> ms alone with the default shape
  chosen = {}   # group -> entry of the fastest shape alone (None: the default)
  cands_of = {}
  for g, ((n_lo, n_hi), grp) in enumerate(groups):
    hb.replan(None)
    db.refresh_plan()
    t_default = _time_group(torch, db, g, stream, reps)
    default[g] = t_default
    ids = hb.order[grp.begin:grp.begin + grp.count]
    status_ref = db.fetch()[0]["status"][ids].copy()
    best = (t_default, None)
    cands = candidates or (CANDIDATES + (SMALL_CANDIDATES if n_hi <= SMALL_N else []))
    cands_of[g] = []
    for nt, lean, onchip in cands:
      entry = {"n_lo": n_lo, "n_hi": n_hi, "block_threads": nt, "lean": lean,
               "onchip": onchip}
      hb.replan([entry])
      db.refresh_plan()
      try:
        t = _time_group(torch, db, g, stream, reps)
      except _lib.QtqpCudaError:
        continue  # the shape does not fit on an SM
      status = db.fetch()[0]["status"][ids]
      if not np.array_equal(status, status_ref):
        continue
      alone[(g, (nt, lean, onchip))] = t
      cands_of[g].append(entry)
      if t < best[0]:
        best = (t, entry)
    chosen[g] = best[1]

  def table_of(sel):
    return [sel[g] for g in sorted(sel) if sel[g] is not None]

  # 256 MiB, larger than the 126 MB L2 of a B200 (the write evicts it).
  flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
  hb.replan(None)
  db.refresh_plan()
  t_batch_default = _time_batch(torch, db, stream, reps, flush)
  status_all = db.fetch()[0]["status"].copy()

  def time_table(sel, r=reps):
    hb.replan(table_of(sel) or None)
    db.refresh_plan()
    try:
      t = _time_batch(torch, db, stream, r, flush)
    except _lib.QtqpCudaError:
      return None
    if not np.array_equal(db.fetch()[0]["status"], status_all):
      return None
    return t

  t_best = time_table(chosen)
  if t_best is None or t_best > t_batch_default:
    chosen = {g: None for g in chosen}
    t_best = t_batch_default
  if batch_pass:
    first = dict(chosen)
    # A change must beat the current table by 2 %, well above the spread of
    # repeated means, so that the pass does not chase noise.
    for g in sorted(default, key=lambda k: -default[k]):
      for entry in cands_of[g]:
        if chosen[g] is not None and entry == chosen[g]:
          continue
        trial = dict(chosen)
        trial[g] = entry
        t = time_table(trial)
        if t is not None and t < 0.98 * t_best:
          chosen, t_best = trial, t
    if chosen != first:
      # The first-stage table against the new one, longer runs, alternated.
      t_first = t_new = 0.0
      for _ in range(2):
        t_first += time_table(first, 2 * reps) or float("inf")
        t_new += time_table(chosen, 2 * reps) or float("inf")
      if t_new >= t_first:
        chosen, t_best = first, t_first / 2
      else:
        t_best = t_new / 2
  table = []
  for g in sorted(chosen):
    e = chosen[g]
    if e is None:
      continue
    key = (e["block_threads"], e["lean"], e["onchip"])
    entry = dict(e)
    entry.update({"ms": round(alone[(g, key)], 4), "default_ms": round(default[g], 4),
                  "batch_ms": round(t_best, 4),
                  "batch_default_ms": round(t_batch_default, 4)})
    table.append(entry)
  hb.replan(None)
  return table


def save(table: list[dict], device=None, path: str | None = None) -> str:
  """Stores the table for this GPU model in the cache file."""
  torch = _lib.require_device()
  path = path or cache_path()
  data = {}
  if os.path.exists(path):
    with open(path) as f:
      data = json.load(f)
  data[_gpu_key(torch, torch.device(device or "cuda"))] = {"dense_batch": table}
  os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
  with open(path, "w") as f:
    json.dump(data, f, indent=1)
  return path


def load(device=None, path: str | None = None) -> list[dict] | None:
  """The cached table for this GPU model, or None."""
  path = path or cache_path()
  if not os.path.exists(path):
    return None
  torch = _lib.require_device()
  with open(path) as f:
    data = json.load(f)
  entry = data.get(_gpu_key(torch, torch.device(device or "cuda")))
  return None if entry is None else entry.get("dense_batch")
