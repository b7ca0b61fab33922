"""Conversion of user arrays to the device carriers the C ABI expects."""
from __future__ import annotations

from typing import Any, Optional

import numpy as np
import torch


def device() -> torch.device:
  if not torch.cuda.is_available():
    raise RuntimeError("ott_b200 needs a CUDA device (sm_100); none is visible")
  return torch.device("cuda", torch.cuda.current_device())


def as_f32(arr: Any, dev: Optional[torch.device] = None) -> torch.Tensor:
  """Contiguous float32 CUDA tensor holding ``arr`` (no copy if it is one)."""
  dev = dev or device()
  if isinstance(arr, torch.Tensor):
    t = arr
  else:
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(arr, dtype=np.float32)))
    if dev.type == "cuda":
      t = t.pin_memory()
  t = t.to(device=dev, dtype=torch.float32, non_blocking=True)
  return t.contiguous()


def stream_handle() -> int:
  return torch.cuda.current_stream().cuda_stream
