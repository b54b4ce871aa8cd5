"""Per-phase time split of one device solve (profiling build).

Usage (on a machine with a B200):

  python -m qtqp_b200.build --phase-timers         # libqtqp_cuda_phase.so
  python -m qtqp_b200.phases batch [--count 4096]  # the 4096 small dense QPs
  python -m qtqp_b200.phases batch --count 1024 --uniform-n 64  # one size
  python -m qtqp_b200.phases large [--n 4096]      # one dense QP, m = 2n
  python -m qtqp_b200.phases sparse [--grid 40]    # one grid-network flow QP
  python -m qtqp_b200.phases sparse_random [--n 6000]
  python -m qtqp_b200.phases mpc [--horizon 100]   # the supernodal path on an MPC QP

The profiling build adds SM-cycle counters around the IPM's phases (thread
0 of every block adds the cycles it spent in a phase); the report divides
them by the SM clock and by the number of blocks of a whole-GPU solve (or of
QPs of a batch), so each figure is the time one block (one QP) spent in that
phase on average.  Without the profiling build the counters stay zero.  The
solve is run once to warm up and once measured.
"""

from __future__ import annotations

import argparse
import ctypes
import os

import numpy as np

from . import _lib
from . import build as _build

PHASES = ["load", "normalize", "gram", "chol", "solve", "residual", "tau", "step", "term",
          "other", "lg_diag", "lg_panel", "lg_trail", "lg_inv", "lg_fwd", "lg_bwd",
          "bp_interior", "bp_chain", "bp_fwd", "bp_chains", "bp_bwd", "cr_stage", "cr_sweep",
          "cr_gemm", "cr_gather", "sn_sub", "sn_top", "sn_fwd_sub", "sn_fwd_top",
          "sn_bwd_top", "sn_bwd_sub", "sn_top_upd", "sn_top_diag", "sn_top_panel",
          "solve_cols", "solve_rows", "inv", "tri"]


def _runner(args):
  """(launch, blocks, result fetch) of the chosen workload."""
  import qtqp_b200 as qb  # pylint: disable=g-import-not-at-top
  from . import batch, large, problems, sparse  # pylint: disable=g-import-not-at-top
  opts = batch.SolveOptions(precision=args.precision)
  if args.workload == "batch":
    if args.uniform_n:
      qps = [qb.QTQP(**dict(zip("abczp", problems.small_dense_instance_n(args.uniform_n, i))))
             for i in range(args.count)]
    else:
      qps = [qb.QTQP(**dict(zip("abczp", problems.small_dense_instance(i))))
             for i in range(args.count)]
    hb = batch.HostBatch(qps, opts, pinned=True)
    db = batch.DeviceBatch(hb, records=False)
    db.upload()
    blocks = sum(g.count for g in hb.plan.groups[:hb.plan.num_groups])
    return db.launch, max(blocks, 1), lambda: db.fetch()[0]
  if args.workload == "large":
    a, b, c, z, p = problems.large_dense(n=args.n, m=2 * args.n, z=args.n // 4)
    dl = large.DeviceLarge(batch.DenseProblem(a=a, b=b, c=c, z=z, p=p), opts, records=False)
    dl.upload()
    return dl.launch, int(_lib.load().qtqp_dense_large_blocks()), lambda: dl.fetch()[0]
  if args.workload == "sparse":
    a, b, c, z, p = problems.grid_flow(args.grid)
  elif args.workload == "sparse_random":
    a, b, c, z, p = problems.sparse_feasible(args.n, args.n, args.n // 10, 4, per_row=2)
  else:
    a, b, c, z, p = problems.mpc_feasible(args.horizon)
  q = qb.QTQP(a=a, b=b, c=c, z=z, p=p)
  plan = q.sparse_plan()
  dg = sparse.DeviceSparseGrid(plan.permuted(q.a, q.b, q.c, q.z, q.p if q.p.nnz else None),
                               plan, opts, records=False)
  dg.upload()
  return dg.launch, int(_lib.load().qtqp_sparse_grid_blocks()), lambda: dg.fetch()[0]


def main(argv=None) -> None:
  ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
  ap.add_argument("workload", choices=["batch", "large", "sparse", "sparse_random", "mpc"])
  ap.add_argument("--count", type=int, default=4096)
  ap.add_argument("--uniform-n", type=int, default=0,
                  help="batch: every QP of this n (m = 2n) instead of n ~ U{8..64}")
  ap.add_argument("--n", type=int, default=None)
  ap.add_argument("--grid", type=int, default=40)
  ap.add_argument("--horizon", type=int, default=100)
  ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
  ap.add_argument("--sm-mhz", type=float, default=1965.0, help="SM clock for cycles -> ms")
  args = ap.parse_args(argv)
  if args.n is None:
    args.n = 4096 if args.workload == "large" else 6000
  if not os.path.exists(_build.PHASE_LIB_PATH):
    raise SystemExit(f"{_build.PHASE_LIB_PATH} is missing: run "
                     "`python -m qtqp_b200.build --phase-timers` first")
  _lib.LIB_PATH = _build.PHASE_LIB_PATH  # before the first load
  import torch  # pylint: disable=g-import-not-at-top
  lib = _lib.load()
  lib.qtqp_phase_cycles.argtypes = [ctypes.c_void_p, ctypes.c_int]
  buf = (ctypes.c_ulonglong * 64)()
  launch, blocks, fetch = _runner(args)
  launch()
  torch.cuda.synchronize()
  lib.qtqp_phase_cycles(buf, 64)  # reads and clears the counters
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record()
  launch()
  e1.record()
  torch.cuda.synchronize()
  lib.qtqp_phase_cycles(buf, 64)
  res = fetch()
  cyc = np.array(buf[:len(PHASES)], dtype=np.float64)
  ms = cyc / (args.sm_mhz * 1e3) / blocks
  print(f"{args.workload}: {e0.elapsed_time(e1):.1f} ms (profiling build), "
        f"iterations {int(np.sum(res['iterations']))}, "
        f"refinement solves {int(np.sum(res['ir_solves']))}")
  # A batch also reports thousands of SM cycles per QP and IPM iteration.
  per_it = (cyc / blocks / max(float(np.mean(res["iterations"])), 1.0) / 1e3
            if args.workload == "batch" else None)
  for k, (name, v) in enumerate(zip(PHASES, ms)):
    if v > 0.005:
      extra = f"  {per_it[k]:8.1f} kcycles per QP-iteration" if per_it is not None else ""
      print(f"  {name:14s} {v:10.2f} ms{extra}")


if __name__ == "__main__":
  main()
