"""ctypes binding of libqtqp_cuda.so (declarations in include/qtqp_cuda.h).

Loading fails loudly: a missing library raises OSError and a machine without a
CUDA device raises ImportError when a backend is instantiated.  There is no
CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqtqp_cuda.so")

QTQP_OK = 0
QTQP_ERR_BAD_ARG = -1
QTQP_ERR_CUDA = -2
QTQP_ERR_NOT_SPD = -3
QTQP_ERR_TIMEOUT = -4
QTQP_ERR_NAN = -5

PREC_FP64 = 0
PREC_MIXED = 1
# qtqp_dense_large_solve flags.
LARGE_HAS_P = 1
LARGE_COLMAJOR = 2

STATS_DOUBLES = 64

# Exported symbols; tests check that the library provides every one of them.
EXPORTS = (
    "qtqp_last_error",
    "qtqp_version",
    "qtqp_device_sm_count",
    "qtqp_host_gather",
    "qtqp_dense_batch_plan",
    "qtqp_dense_batch_plan_tuned",
    "qtqp_dense_batch_solve",
    "qtqp_dense_batch_solve_from",
    "qtqp_dense_batch_solve_group",
    "qtqp_dense_batch_noalloc_max_workspace",
    "qtqp_dense_batch_solve_noalloc",
    "qtqp_band_batch_plan",
    "qtqp_band_batch_solve",
    "qtqp_kkt_dense_workspace_bytes",
    "qtqp_kkt_dense_set",
    "qtqp_kkt_dense_factorize",
    "qtqp_kkt_dense_solve",
    "qtqp_kkt_dense_matvec",
    "qtqp_dense_equilibrate",
    "qtqp_mlp_gemm",
    "qtqp_mlp_relu_grad",
    "qtqp_mlp_colsum",
    "qtqp_mlp_mse_grad",
    "qtqp_mlp_hinge_grad",
    "qtqp_mlp_gemm_bf16",
    "qtqp_mlp_to_bf16",
    "qtqp_mlp_adam",
    "qtqp_mlp_decode",
    "qtqp_dense_large_workspace_bytes",
    "qtqp_dense_large_blocks",
    "qtqp_dense_large_solve",
    "qtqp_tc_split_tf32",
    "qtqp_tc_gram_f32",
    "qtqp_band_grid_default_parts",
    "qtqp_band_grid_workspace_bytes",
    "qtqp_band_grid_solve",
    "qtqp_wait_selftest_workspace_bytes",
    "qtqp_wait_selftest",
    "qtqp_sparse_analyze",
    "qtqp_sparse_export",
    "qtqp_sparse_free",
    "qtqp_sparse_grid_blocks",
    "qtqp_sparse_grid_workspace_bytes",
    "qtqp_sparse_grid_solve",
)


class Options(ctypes.Structure):
  _fields_ = [
      ("atol", ctypes.c_double),
      ("rtol", ctypes.c_double),
      ("atol_infeas", ctypes.c_double),
      ("rtol_infeas", ctypes.c_double),
      ("step_size_scale", ctypes.c_double),
      ("min_static_regularization", ctypes.c_double),
      ("linear_solver_atol", ctypes.c_double),
      ("linear_solver_rtol", ctypes.c_double),
      ("max_iter", ctypes.c_int32),
      ("max_iterative_refinement_steps", ctypes.c_int32),
      ("equilibrate", ctypes.c_int32),
      ("precision", ctypes.c_int32),
      ("collect_stats", ctypes.c_int32),
      ("tau_mode", ctypes.c_int32),
      ("warm_corrections", ctypes.c_int32),
      ("warm_shift", ctypes.c_double),
  ]


class DenseInstance(ctypes.Structure):
  _fields_ = [
      ("n", ctypes.c_int32),
      ("m", ctypes.c_int32),
      ("z", ctypes.c_int32),
      ("has_p", ctypes.c_int32),
      ("a_off", ctypes.c_int64),
      ("p_off", ctypes.c_int64),
      ("n_off", ctypes.c_int64),
      ("m_off", ctypes.c_int64),
      ("ws_off", ctypes.c_int64),
      ("st_off", ctypes.c_int64),
  ]


class Result(ctypes.Structure):
  _fields_ = [
      ("status", ctypes.c_int32),
      ("iterations", ctypes.c_int32),
      ("error", ctypes.c_int32),
      ("fp32_factorizations", ctypes.c_int32),
      ("fp64_factorizations", ctypes.c_int32),
      ("ir_solves", ctypes.c_int32),
      ("warm_started", ctypes.c_int32),
      ("reserved", ctypes.c_int32),
      ("tau", ctypes.c_double),
      ("pcost", ctypes.c_double),
      ("dcost", ctypes.c_double),
      ("pres", ctypes.c_double),
      ("dres", ctypes.c_double),
      ("gap", ctypes.c_double),
  ]


MAX_GROUPS = 8


class LaunchGroup(ctypes.Structure):
  _fields_ = [("begin", ctypes.c_int32), ("count", ctypes.c_int32),
              ("block_threads", ctypes.c_int32), ("smem_bytes", ctypes.c_int32),
              ("slots", ctypes.c_int32), ("lean", ctypes.c_int32),
              ("slot_off", ctypes.c_uint64), ("slot_bytes", ctypes.c_uint64)]


class BatchTuning(ctypes.Structure):
  _fields_ = [("n_lo", ctypes.c_int32), ("n_hi", ctypes.c_int32),
              ("block_threads", ctypes.c_int32), ("lean", ctypes.c_int32),
              ("onchip", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class BatchPlan(ctypes.Structure):
  _fields_ = [("num_groups", ctypes.c_int32), ("reserved", ctypes.c_int32),
              ("groups", LaunchGroup * MAX_GROUPS), ("workspace_bytes", ctypes.c_uint64)]


# numpy views of the same layouts (for bulk packing / unpacking).
INSTANCE_DTYPE = np.dtype([(name, np.int32 if ct is ctypes.c_int32 else np.int64)
                           for name, ct in DenseInstance._fields_])
RESULT_DTYPE = np.dtype([(name, np.int32 if ct is ctypes.c_int32 else np.float64)
                         for name, ct in Result._fields_])
assert INSTANCE_DTYPE.itemsize == ctypes.sizeof(DenseInstance)
assert RESULT_DTYPE.itemsize == ctypes.sizeof(Result)

_lock = threading.Lock()
_lib = None


class QtqpCudaError(RuntimeError):
  """A C-ABI call returned an error code."""

  def __init__(self, code: int, msg: str):
    super().__init__(f"libqtqp_cuda error {code}: {msg}")
    self.code = code


def load() -> ctypes.CDLL:
  """Loads the library (building nothing); raises OSError when it is absent."""
  global _lib
  with _lock:
    if _lib is not None:
      return _lib
    if not os.path.exists(LIB_PATH):
      raise OSError(
          f"{LIB_PATH} is missing: build it with `python -m qtqp_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
    lib.qtqp_last_error.restype = ctypes.c_char_p
    lib.qtqp_version.restype = ctypes.c_int
    lib.qtqp_device_sm_count.restype = ctypes.c_int
    lib.qtqp_host_gather.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]
    lib.qtqp_dense_batch_plan.argtypes = [vp, i32, ctypes.POINTER(Options), vp, i32, i32,
                                          ctypes.POINTER(BatchPlan)]
    lib.qtqp_dense_batch_plan_tuned.argtypes = [vp, i32, ctypes.POINTER(Options), vp, vp, i32,
                                                ctypes.POINTER(BatchPlan)]
    lib.qtqp_dense_batch_solve.argtypes = [vp, vp, ctypes.POINTER(BatchPlan), vp, vp, vp, vp,
                                           vp, vp, vp, vp, vp, vp, sz,
                                           ctypes.POINTER(Options), vp]
    lib.qtqp_dense_batch_solve_from.argtypes = [vp, vp, ctypes.POINTER(BatchPlan), vp, vp, vp,
                                                vp, vp, vp, vp, vp, vp, vp, sz,
                                                ctypes.POINTER(Options), vp, vp, vp, vp]
    lib.qtqp_dense_batch_solve_group.argtypes = [vp, vp, ctypes.POINTER(BatchPlan), i32, vp, vp,
                                                 vp, vp, vp, vp, vp, vp, vp, vp, sz,
                                                 ctypes.POINTER(Options), vp]
    lib.qtqp_dense_batch_noalloc_max_workspace.restype = sz
    lib.qtqp_dense_batch_noalloc_max_workspace.argtypes = []
    lib.qtqp_dense_batch_solve_noalloc.argtypes = [vp, vp, ctypes.POINTER(BatchPlan), vp, vp,
                                                   vp, vp, vp, vp, vp, vp, vp,
                                                   ctypes.POINTER(Options), vp]
    lib.qtqp_band_batch_plan.argtypes = [vp, i32, ctypes.POINTER(Options), i32, vp,
                                         ctypes.POINTER(BatchPlan)]
    lib.qtqp_band_batch_solve.argtypes = [vp, vp, ctypes.POINTER(BatchPlan), vp, vp, vp, vp,
                                          vp, vp, vp, vp, vp, vp, sz,
                                          ctypes.POINTER(Options), vp, vp, vp, vp]
    f32, f64, i64 = ctypes.c_float, ctypes.c_double, ctypes.c_int64
    lib.qtqp_mlp_gemm.argtypes = [i32, i32, i32, f32, vp, i32, i32, vp, i32, i32, f32, vp, i32,
                                  vp, i32, vp]
    lib.qtqp_mlp_relu_grad.argtypes = [vp, vp, i64, vp]
    lib.qtqp_mlp_colsum.argtypes = [vp, i32, i32, vp, vp]
    lib.qtqp_mlp_mse_grad.argtypes = [vp, vp, i64, vp, vp, vp]
    lib.qtqp_mlp_hinge_grad.argtypes = [vp, vp, i32, i32, i32, vp, f32, f32, vp, vp, vp]
    lib.qtqp_mlp_gemm_bf16.argtypes = [i32, i32, i32, vp, vp, vp, i32, vp, i32, vp, i32, vp, vp]
    lib.qtqp_mlp_to_bf16.argtypes = [vp, i32, i32, i32, vp, vp]
    lib.qtqp_mlp_adam.argtypes = [vp, vp, vp, vp, i64, f32, f32, f32, f32, i32, vp]
    lib.qtqp_mlp_decode.argtypes = [vp, vp, vp, i32, i32, i32, i32, f64, vp, vp, vp, vp]
    lib.qtqp_dense_large_workspace_bytes.restype = sz
    lib.qtqp_dense_large_workspace_bytes.argtypes = [i32, i32]
    lib.qtqp_dense_large_blocks.restype = i32
    lib.qtqp_dense_large_blocks.argtypes = []
    lib.qtqp_dense_large_solve.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp,
                                           vp, vp, sz, ctypes.POINTER(Options), vp]
    lib.qtqp_band_grid_default_parts.restype = i32
    lib.qtqp_band_grid_default_parts.argtypes = [vp]
    lib.qtqp_band_grid_workspace_bytes.restype = sz
    lib.qtqp_band_grid_workspace_bytes.argtypes = [vp, i32]
    lib.qtqp_band_grid_solve.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz,
                                         ctypes.POINTER(Options), vp]
    lib.qtqp_tc_split_tf32.argtypes = [vp, i64, vp, vp, vp]
    lib.qtqp_wait_selftest_workspace_bytes.restype = sz
    lib.qtqp_wait_selftest_workspace_bytes.argtypes = []
    lib.qtqp_wait_selftest.argtypes = [i32, i32, i32, ctypes.c_uint32, vp, vp, vp]
    lib.qtqp_tc_gram_f32.argtypes = [i32, i32, vp, vp, i32, vp, i32, i32, vp, vp]
    lib.qtqp_kkt_dense_workspace_bytes.restype = sz
    lib.qtqp_kkt_dense_workspace_bytes.argtypes = [i32, i32]
    lib.qtqp_kkt_dense_set.argtypes = [i32, i32, vp, vp, vp, vp]
    lib.qtqp_kkt_dense_factorize.argtypes = [i32, i32, vp, i32, vp, vp, vp]
    lib.qtqp_kkt_dense_solve.argtypes = [i32, i32, vp, vp, vp, vp]
    lib.qtqp_kkt_dense_matvec.argtypes = [i32, i32, vp, vp, vp, vp]
    lib.qtqp_dense_equilibrate.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.qtqp_sparse_analyze.argtypes = [i32, i32, vp, vp, vp, vp, i32, i32,
                                        ctypes.POINTER(vp), ctypes.POINTER(SparseDesc)]
    lib.qtqp_sparse_export.argtypes = [vp, ctypes.POINTER(SparseDesc), vp, vp, vp]
    lib.qtqp_sparse_free.restype = None
    lib.qtqp_sparse_free.argtypes = [vp]
    lib.qtqp_sparse_grid_blocks.restype = i32
    lib.qtqp_sparse_grid_blocks.argtypes = []
    lib.qtqp_sparse_grid_workspace_bytes.restype = sz
    lib.qtqp_sparse_grid_workspace_bytes.argtypes = [vp, ctypes.POINTER(SparseDesc)]
    lib.qtqp_sparse_grid_solve.argtypes = [vp, ctypes.POINTER(SparseDesc), vp, vp, vp, vp, vp,
                                           vp, vp, vp, vp, vp, vp, vp, sz,
                                           ctypes.POINTER(Options), vp]
    for name in EXPORTS:  # every declared entry point must resolve
      getattr(lib, name)
    _lib = lib
    return lib


def check(rc: int) -> None:
  if rc != QTQP_OK:
    msg = load().qtqp_last_error()
    raise QtqpCudaError(rc, msg.decode() if msg else "")


def require_device():
  """Returns torch with a visible CUDA device, else raises ImportError."""
  import torch  # pylint: disable=g-import-not-at-top
  if not torch.cuda.is_available():
    raise ImportError("qtqp_b200: no CUDA device is visible (the CUDA backend "
                      "has no CPU fallback)")
  load()
  return torch


def stream_handle(torch_stream) -> int:
  return int(torch_stream.cuda_stream)


class BandInstance(ctypes.Structure):
  _fields_ = [("n", ctypes.c_int32), ("m", ctypes.c_int32), ("z", ctypes.c_int32),
              ("has_p", ctypes.c_int32), ("bw", ctypes.c_int32), ("nnz_a", ctypes.c_int32),
              ("nnz_p", ctypes.c_int32), ("reserved", ctypes.c_int32),
              ("a_ptr", ctypes.c_int64), ("a_idx", ctypes.c_int64), ("a_val", ctypes.c_int64),
              ("at_ptr", ctypes.c_int64), ("at_idx", ctypes.c_int64),
              ("at_val", ctypes.c_int64), ("p_ptr", ctypes.c_int64),
              ("p_idx", ctypes.c_int64), ("p_val", ctypes.c_int64),
              ("n_off", ctypes.c_int64), ("m_off", ctypes.c_int64), ("st_off", ctypes.c_int64)]


BAND_DTYPE = np.dtype([(name, np.int32 if ct is ctypes.c_int32 else np.int64)
                       for name, ct in BandInstance._fields_])
assert BAND_DTYPE.itemsize == ctypes.sizeof(BandInstance)


class SparseDesc(ctypes.Structure):
  """qtqp_sparse_desc: sizes and pool offsets of a supernodal symbolic plan."""
  _fields_ = ([(f, ctypes.c_int32) for f in ("n", "nsuper", "blocks", "top_levels", "max_rows",
                                              "max_width", "tree_levels", "reserved")] +
              [(f, ctypes.c_int64) for f in ("nvals", "ngram", "nrows", "nupd", "nranges",
                                              "ntop", "nnz_l", "top_row_slabs")] +
              [("flops", ctypes.c_double)] +
              [(f, ctypes.c_int64) for f in ("o_first", "o_colsn", "o_rows", "o_upd_ptr",
                                              "o_upd_src", "o_upd_off", "o_upd_cnt",
                                              "o_cta_ptr", "o_cta_range", "o_top_ptr",
                                              "o_top_list", "o_top_slab", "o_gcol", "o_grow",
                                              "o_rowptr",
                                              "o_valptr", "o_gpos", "n32", "n64")])
