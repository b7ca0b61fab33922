from ott_b200.problems.linear import linear_problem  # noqa: F401
