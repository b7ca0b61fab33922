from ott_b200.problems import linear  # noqa: F401
