"""``qtqp.direct``: the KKT plugin interface (src/qtqp/direct.py:49-109) and
the CUDA backend, re-exported from ``qtqp_b200.direct``."""

from qtqp_b200.direct import *  # noqa: F401,F403  pylint: disable=wildcard-import
from qtqp_b200.direct import CudaDenseSolver, LinearSolver, diag_data_indices  # noqa: F401
