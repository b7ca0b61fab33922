from ott_b200.initializers.neural import meta_initializer  # noqa: F401
