"""The JSON line contract of bench.py's reference arm (CPU only).

`bench.py --impl reference` times the oracle port of the reference algorithm
on the host cores; it needs no GPU, so its line is checked here for each
workload (at reduced sizes): one JSON object with the metric, unit, timing,
config, cpu_baseline and e2e keys, and silence (exit 0, no line) on ranks
other than 0.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run_bench(extra_env=None, *args):
  env = dict(os.environ)
  env.update(extra_env or {})
  return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                        cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


WORKLOADS = {
    "batch_small": [],
    "dense_large": ["--workload", "dense_large", "--large-n", "64"],
    "mpc": ["--workload", "mpc", "--mpc-horizon", "20"],
    "parametric": ["--workload", "parametric", "--train", "64", "--count", "16"],
    "sparse": ["--workload", "sparse", "--grid", "8"],
}


@pytest.mark.parametrize("workload", sorted(WORKLOADS))
def test_reference_arm_line(workload):
  proc = _run_bench({"RANK": "0", "WORLD_SIZE": "1"}, *WORKLOADS[workload], "--impl",
                    "reference", "--steps", "1", "--warmup", "1")
  assert proc.returncode == 0, proc.stderr[-2000:]
  lines = [l for l in proc.stdout.splitlines() if l.startswith("{")]
  assert len(lines) == 1, proc.stdout
  rec = json.loads(lines[0])
  for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
    assert key in rec, key
  assert rec["impl"] == "reference"
  assert rec["unit"] == "QPs/s" and rec["higher_is_better"] is True
  assert rec["steps"] == 1 and rec["warmup"] == 1 and rec["n_gpus"] == 1
  assert rec["value"] > 0 and rec["ms_per_step"] > 0
  assert rec["vs_baseline"] is None
  assert "workload" in rec["config"]
  cpu = rec["cpu_baseline"]
  assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == rec["value"]
  assert cpu["sample"]
  e2e = rec["e2e"]
  assert e2e["value"] == rec["value"] and e2e["unit"] == rec["unit"]
  assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


@pytest.mark.parametrize("workload", sorted(WORKLOADS))
def test_reference_arm_other_ranks_are_silent(workload):
  proc = _run_bench({"RANK": "1", "WORLD_SIZE": "4"}, *WORKLOADS[workload], "--impl",
                    "reference", "--steps", "1", "--warmup", "0")
  assert proc.returncode == 0, proc.stderr[-2000:]
  assert not [l for l in proc.stdout.splitlines() if l.startswith("{")]
