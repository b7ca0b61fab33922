from ott_b200.solvers.linear import sinkhorn  # noqa: F401
from ott_b200.solvers.linear._solve import solve, solve_batch  # noqa: F401

__all__ = ["sinkhorn", "solve", "solve_batch"]
