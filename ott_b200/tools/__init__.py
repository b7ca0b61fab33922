from ott_b200.tools import sinkhorn_divergence  # noqa: F401

__all__ = ["sinkhorn_divergence"]
