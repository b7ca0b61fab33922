from ott_b200.solvers.linear import acceleration, annealing, implicit_differentiation, sinkhorn  # noqa: F401
from ott_b200.solvers.linear._solve import reg_ot_cost, solve, solve_batch  # noqa: F401

__all__ = ["acceleration", "annealing", "implicit_differentiation", "reg_ot_cost", "sinkhorn",
           "solve", "solve_batch"]
