"""Sinkhorn initializers (ott/initializers/linear/initializers.py:30-131).

The initializer slot: ``init_fu`` / ``init_gv`` return initial potentials;
``__call__`` masks them with ``-inf`` where the weight is zero (:95-98).
The default initializer is applied inside the solve kernel itself (zeros,
masked), so it costs no extra launch.
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch


class SinkhornInitializer:
  """Base class; subclasses define ``init_fu`` and ``init_gv``."""

  def init_fu(self, ot_prob, lse_mode: bool, rng=None) -> Optional[torch.Tensor]:
    raise NotImplementedError

  def init_gv(self, ot_prob, lse_mode: bool, rng=None) -> Optional[torch.Tensor]:
    raise NotImplementedError

  def __call__(self, ot_prob, lse_mode: bool = True, rng=None
               ) -> Tuple[Optional[torch.Tensor], Optional[torch.Tensor]]:
    """Initial (f, g); ``None`` entries mean "zeros", masked on the device."""
    if not lse_mode:
      raise NotImplementedError("kernel mode (lse_mode=False) is not on this path")
    return (self.init_fu(ot_prob, lse_mode, rng), self.init_gv(ot_prob, lse_mode, rng))


class DefaultInitializer(SinkhornInitializer):
  """Zeros, ``-inf`` at zero weights (:112-131). Returns ``None`` so the
  solve kernel writes them directly."""

  def init_fu(self, ot_prob, lse_mode: bool, rng=None):
    return None

  def init_gv(self, ot_prob, lse_mode: bool, rng=None):
    return None
