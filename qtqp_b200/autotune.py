"""Autotuner of the dense batch's launch shapes (no reference counterpart).

The batch solve runs one persistent launch per size class of the instances
(qtqp_dense_batch_plan); how fast a class solves depends on its launch
shape: threads per block, the register-capped ("lean") or unrestricted
kernel, and whether A and P stay in shared memory or are read through L2.
The default plan chooses by heuristics.  tune_dense_batch times every
candidate shape on each launch group of a representative batch, on the
device (CUDA events, each group launched alone), keeps the fastest, and
returns a table of {n_lo, n_hi, block_threads, lean, onchip} entries that
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


def tune_dense_batch(problems, opts: _batch.SolveOptions | None = None, candidates=None,
                     reps: int = 3, device=None) -> list[dict]:
  """Times each candidate (block_threads, lean, onchip) on every launch group
  of the default plan of `problems` and returns the tuning table of the
  fastest shapes (ms of the default and the chosen shape in each entry).  A
  candidate that changes any instance's status against the default shape is
  never chosen."""
  torch = _lib.require_device()
  opts = opts or _batch.SolveOptions()
  dev = torch.device(device or "cuda")
  stream = torch.cuda.current_stream(dev)
  hb = _batch.HostBatch(problems, opts, pinned=True)
  db = _batch.DeviceBatch(hb, device=dev, records=False)
  db.upload(stream)
  groups = [(hb.group_n_range(g), hb.plan.groups[g]) for g in range(hb.plan.num_groups)]
  table = []
  for g, ((n_lo, n_hi), grp) in enumerate(groups):
    hb.replan(None)
    db.refresh_plan()
    t_default = _time_group(torch, db, g, stream, reps)
    ids = hb.order[grp.begin:grp.begin + grp.count]
    status_ref = db.fetch()[0]["status"][ids].copy()
    best = (t_default, None)
    cands = candidates or (CANDIDATES + (SMALL_CANDIDATES if n_hi <= SMALL_N else []))
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
      if t < best[0]:
        best = (t, entry)
    if best[1] is not None:
      entry = dict(best[1])
      entry.update({"ms": round(best[0], 4), "default_ms": round(t_default, 4)})
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
