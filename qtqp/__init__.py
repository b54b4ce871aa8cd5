"""``qtqp``: the B200 build under the reference's own package name.

Code written against google-deepmind/qtqp keeps its imports and calls:

    import qtqp
    sol = qtqp.QTQP(a=a, b=b, c=c, z=z, p=p).solve(
        linear_solver=qtqp.LinearSolver.CUDA)

Everything here is the ``qtqp_b200`` package (the device-resident interior-
point method behind the C-ABI library); this module only re-exports it under
the name the reference's users import.
"""

from qtqp_b200 import (LinearSolver, QTQP, Solution, SolutionStatus, __version__, direct,
                       solve_batch)

__all__ = ["QTQP", "Solution", "SolutionStatus", "LinearSolver", "solve_batch", "direct",
           "__version__"]
