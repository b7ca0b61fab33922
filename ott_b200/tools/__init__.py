from ott_b200.tools import segment_sinkhorn, sinkhorn_divergence  # noqa: F401

__all__ = ["segment_sinkhorn", "sinkhorn_divergence"]
