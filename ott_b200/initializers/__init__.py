from ott_b200.initializers import linear, neural  # noqa: F401
