"""Readers of the golden fixtures written by tests/golden/make_golden.py."""

import functools
import os

import numpy as np
import scipy.sparse as sp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@functools.lru_cache(maxsize=None)
def load(name: str):
  with np.load(os.path.join(GOLDEN, name), allow_pickle=False) as f:
    return {k: f[k] for k in f.files}


def csc(d, prefix):
  shape = tuple(int(v) for v in d[prefix + "_shape"])
  return sp.csc_matrix((d[prefix + "_data"], d[prefix + "_indices"], d[prefix + "_indptr"]),
                       shape=shape)


def e2e_names():
  return [str(n) for n in load("reference_e2e.npz")["names"]]


def e2e_problem(name):
  d = load("reference_e2e.npz")
  return (csc(d, name + "/a"), d[name + "/b"], d[name + "/c"], int(d[name + "/z"]),
          csc(d, name + "/p"))


def e2e_result(name, backend="SCIPY", eq=True):
  d = load("reference_e2e.npz")
  tag = f"{name}/{backend}/{'eq' if eq else 'noeq'}"
  if tag + "/status" not in d:
    return None
  keys = ("x", "y", "s", "mu", "sigma", "alpha", "tau", "pres", "dres", "gap", "pcost")
  out = {k: d[tag + "/" + k] for k in keys}
  out["status"] = str(d[tag + "/status"])
  out["iters"] = int(d[tag + "/iters"])
  return out
