from ott_b200.solvers.linear import annealing, sinkhorn  # noqa: F401
from ott_b200.solvers.linear._solve import reg_ot_cost, solve, solve_batch  # noqa: F401

__all__ = ["annealing", "reg_ot_cost", "sinkhorn", "solve", "solve_batch"]
