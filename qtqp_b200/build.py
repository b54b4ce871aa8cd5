"""Builds libqtqp_cuda.so in-tree with nvcc for sm_100a (B200).

Usage: python -m qtqp_b200.build [--debug]

The library is a plain C-ABI shared object (include/qtqp_cuda.h); it does not
link against PyTorch.  The build is incremental on source mtimes.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
_CSRC = os.path.join(_HERE, "csrc")
_INC = os.path.join(_ROOT, "include")
LIB_PATH = os.path.join(_HERE, "libqtqp_cuda.so")
# The profiling build: per-phase SM-cycle counters (-DQTQP_PHASE_TIMERS, read
# with qtqp_phase_cycles; qtqp_b200.phases reports them).
PHASE_LIB_PATH = os.path.join(_HERE, "libqtqp_cuda_phase.so")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
  cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
  if not os.path.exists(cand):
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
  return cand


def sources() -> list[str]:
  return sorted(os.path.join(_CSRC, f) for f in os.listdir(_CSRC) if f.endswith(".cu"))


def _deps() -> list[str]:
  files = sources()
  files += [os.path.join(_CSRC, f) for f in os.listdir(_CSRC) if f.endswith((".cuh", ".h"))]
  files += [os.path.join(_INC, f) for f in os.listdir(_INC) if f.endswith(".h")]
  return files


def up_to_date(path: str = LIB_PATH) -> bool:
  if not os.path.exists(path):
    return False
  t = os.path.getmtime(path)
  return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, debug: bool = False, verbose: bool = False,
          phase_timers: bool = False) -> str:
  """Compiles every .cu under csrc/ (in parallel) into libqtqp_cuda.so, or,
  with phase_timers, into the profiling build libqtqp_cuda_phase.so (per-phase
  cycle counters; relocatable device code, since the counters are one device
  array shared by every kernel)."""
  out = PHASE_LIB_PATH if phase_timers else LIB_PATH
  if not force and not debug and up_to_date(out):
    return out
  import concurrent.futures
  import tempfile
  common = [_nvcc(), *ARCH_FLAGS, "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-I", _INC, "-I", _CSRC, "--expt-relaxed-constexpr"]
  common += ["-O0", "-G"] if debug else ["-O3"]
  if phase_timers:
    common += ["-DQTQP_PHASE_TIMERS", "-rdc=true"]
  if verbose:
    common += ["-Xptxas", "-v"]
  with tempfile.TemporaryDirectory(prefix="qtqp_build_") as tmp:
    def compile_one(src):
      obj = os.path.join(tmp, os.path.basename(src) + ".o")
      proc = subprocess.run([*common, "-c", src, "-o", obj], capture_output=True, text=True)
      return src, obj, proc
    objs = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
      for src, obj, proc in ex.map(compile_one, sources()):
        if proc.returncode != 0:
          raise RuntimeError(f"nvcc failed on {src}:\n{proc.stderr}\n{proc.stdout}")
        if verbose:
          sys.stderr.write(proc.stderr)
        objs.append(obj)
    link = [_nvcc(), *ARCH_FLAGS, *(["-rdc=true"] if phase_timers else []), "-shared", "-o",
            out + ".tmp", *objs]
    proc = subprocess.run(link, capture_output=True, text=True)
    if proc.returncode != 0:
      raise RuntimeError(f"nvcc link failed:\n{proc.stderr}\n{proc.stdout}")
  os.replace(out + ".tmp", out)
  return out


if __name__ == "__main__":
  print(build(force=True, debug="--debug" in sys.argv, verbose="-v" in sys.argv,
              phase_timers="--phase-timers" in sys.argv))
