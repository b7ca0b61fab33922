"""Epsilon scheduler (ott/geometry/epsilon_scheduler.py:22-73)."""
from typing import Optional

#: Scaling applied to a statistic (mean/std) of the cost for the default
#: epsilon (epsilon_scheduler.py:22).
DEFAULT_EPSILON_SCALE = 0.05


class Epsilon:
  """``epsilon(it) = max(init * decay**it, 1) * target``."""

  def __init__(self, target: float, init: float = 1.0, decay: float = 1.0):
    assert decay <= 1.0, f"Decay must be <= 1, found {decay}."
    self.target = target
    self.init = init
    self.decay = decay

  def __call__(self, it: Optional[int]) -> float:
    if it is None:
      return self.target
    return max(self.init * (self.decay ** it), 1.0) * self.target

  def __repr__(self) -> str:
    return (f"{self.__class__.__name__}(target={self.target:.4f}, "
            f"init={self.init:.4f}, decay={self.decay:.4f})")
