"""Geometry base: epsilon resolution (ott/geometry/geometry.py:30-176)."""
from __future__ import annotations

from typing import Literal, Optional, Union

from ott_b200.geometry import epsilon_scheduler as eps_scheduler


class Geometry:
  """Holds the regularisation settings shared by every geometry.

  ``epsilon`` / ``relative_epsilon`` follow geometry.py:148-176:
  ``epsilon=None, relative_epsilon=None`` gives ``0.05 * std(C)``; a float
  with ``relative_epsilon=None`` is used as is; otherwise ``epsilon`` (default
  0.05) multiplies ``mean(C)`` or ``std(C)``.
  """

  def __init__(
      self,
      epsilon: Optional[Union[float, eps_scheduler.Epsilon]] = None,
      relative_epsilon: Optional[Literal["mean", "std"]] = None,
      scale_cost: Union[float, str] = 1.0,
  ):
    self._epsilon_init = epsilon
    self._relative_epsilon = relative_epsilon
    self._scale_cost = scale_cost
    self._eps_cache: Optional[eps_scheduler.Epsilon] = None

  # statistics supplied by subclasses
  @property
  def mean_cost_matrix(self) -> float:
    raise NotImplementedError

  @property
  def std_cost_matrix(self) -> float:
    raise NotImplementedError

  @property
  def epsilon_scheduler(self) -> eps_scheduler.Epsilon:
    """geometry.py:148-171."""
    if self._eps_cache is not None:
      return self._eps_cache
    if isinstance(self._epsilon_init, eps_scheduler.Epsilon):
      sched = self._epsilon_init
    elif self._relative_epsilon is None:
      if self._epsilon_init is not None:
        sched = eps_scheduler.Epsilon(float(self._epsilon_init))
      else:
        sched = eps_scheduler.Epsilon(
            target=eps_scheduler.DEFAULT_EPSILON_SCALE * self.std_cost_matrix)
    else:
      if self._relative_epsilon == "std":
        scale = self.std_cost_matrix
      elif self._relative_epsilon == "mean":
        scale = self.mean_cost_matrix
      else:
        raise ValueError(f"Invalid relative epsilon: {self._relative_epsilon}.")
      mult = (eps_scheduler.DEFAULT_EPSILON_SCALE
              if self._epsilon_init is None else float(self._epsilon_init))
      sched = eps_scheduler.Epsilon(target=mult * scale)
    self._eps_cache = sched
    return sched

  @property
  def epsilon(self) -> float:
    """Target epsilon (geometry.py:173-176)."""
    return self.epsilon_scheduler.target
