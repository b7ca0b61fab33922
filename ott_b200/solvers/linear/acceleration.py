"""Momentum settings of the Sinkhorn update (ott/solvers/linear/acceleration.py:
126-172). The solver runs weight 1 (the default) for every problem, and weight
1/2 from iteration 0 with parallel updates for symmetric problems (x = y,
a = b), the setting the reference's Sinkhorn divergence uses for its x/x and
y/y terms; adaptive momentum is not on this path."""
from __future__ import annotations

import dataclasses
import math


@dataclasses.dataclass(frozen=True)
class Momentum:
  """acceleration.py:126-137: ``start``, ``error_threshold``, ``value``,
  ``inner_iterations`` (the weight is ``value`` from ``start`` on)."""
  start: int = 0
  error_threshold: float = math.inf
  value: float = 1.0
  inner_iterations: int = 1
