from ott_b200.initializers.linear import initializers  # noqa: F401
