from ott_b200.solvers import linear  # noqa: F401
