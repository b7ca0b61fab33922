"""ott_b200: log-domain Sinkhorn on squared-Euclidean point clouds for B200.

A drop-in for the hot path of ott-jax's ``ott.solvers.linear.solve`` /
``sinkhorn.Sinkhorn(lse_mode=True)`` on ``PointCloud(cost_fn=SqEuclidean())``.
The module layout mirrors ott's (``geometry``, ``problems.linear``,
``solvers.linear``, ``initializers``); arrays are torch CUDA tensors. All
arithmetic runs in the sm_100a kernels of ``libottb200.so`` behind the C ABI
in ``include/ott_b200.h``.
"""
from ott_b200 import geometry, initializers, problems, solvers  # noqa: F401

__version__ = "0.1.0"
