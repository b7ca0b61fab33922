"""Linear OT problem (ott/problems/linear/linear_problem.py:31-107)."""
from __future__ import annotations

from typing import Any, Optional

import torch

from ott_b200 import _arrays


class LinearProblem:
  """Geometry plus marginals; ``a``/``b`` default to uniform (:66-79)."""

  def __init__(self, geom, a: Optional[Any] = None, b: Optional[Any] = None,
               tau_a: float = 1.0, tau_b: float = 1.0):
    self.geom = geom
    dev = geom.x.device
    n, m = geom.shape
    self._a = None if a is None else _arrays.as_f32(a, dev)
    self._b = None if b is None else _arrays.as_f32(b, dev)
    if self._a is not None and tuple(self._a.shape) != (n,):
      raise ValueError(f"a must have shape ({n},), got {tuple(self._a.shape)}")
    if self._b is not None and tuple(self._b.shape) != (m,):
      raise ValueError(f"b must have shape ({m},), got {tuple(self._b.shape)}")
    self.tau_a = tau_a
    self.tau_b = tau_b
    # the uniform defaults, made once; _a / _b stay None so that
    # is_uniform keeps telling whether weights were passed
    self._a_uniform: Optional[torch.Tensor] = None
    self._b_uniform: Optional[torch.Tensor] = None

  @property
  def a(self) -> torch.Tensor:
    if self._a is not None:
      return self._a
    if self._a_uniform is None:
      n, _ = self.geom.shape
      self._a_uniform = torch.full((n,), 1.0 / n, dtype=torch.float32,
                                   device=self.geom.x.device)
    return self._a_uniform

  @property
  def b(self) -> torch.Tensor:
    if self._b is not None:
      return self._b
    if self._b_uniform is None:
      _, m = self.geom.shape
      self._b_uniform = torch.full((m,), 1.0 / m, dtype=torch.float32,
                                   device=self.geom.x.device)
    return self._b_uniform

  @property
  def is_balanced(self) -> bool:
    return self.tau_a == 1.0 and self.tau_b == 1.0

  @property
  def is_uniform(self) -> bool:
    return self._a is None and self._b is None

  @property
  def is_equal_size(self) -> bool:
    return self.geom.shape[0] == self.geom.shape[1]

  @property
  def is_assignment(self) -> bool:
    return self.is_equal_size and self.is_uniform and self.is_balanced

  @property
  def epsilon(self) -> float:
    return self.geom.epsilon

  @property
  def dtype(self):
    return self.geom.dtype
