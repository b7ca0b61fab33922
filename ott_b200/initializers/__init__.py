from ott_b200.initializers import linear  # noqa: F401
