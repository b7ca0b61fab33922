"""Progress callbacks for ``Sinkhorn(progress_fn=...)`` (ott/utils.py:105-231).

The callbacks receive ``(iteration, inner_iterations, max_iterations,
state)`` with ``state.errors`` the errors buffer so far (-1 where a block
has not been reached). The solver calls them while its persistent launch
runs, once per error block as the block ends (the iterations
``inner_iterations - 1``, ``2 inner_iterations - 1``, ...), which are the
calls on which these callbacks act in the reference too; the kernel writes
each block's error into pinned host memory, which the calling thread polls.
"""
from __future__ import annotations

import io
from typing import Any, Callable, Optional, Tuple

import numpy as np

__all__ = ["default_progress_fn", "tqdm_progress_fn"]

IOStatus = Tuple[Any, Any, Any, Any]


def _prepare_info(status: IOStatus) -> Tuple[int, int, int, np.ndarray]:
  """utils.py:224-231: 1-based iteration, inner iterations, total, errors."""
  iteration, inner_iterations, total_iter, state = status
  errors = state.errors
  errors = (errors.detach().cpu().numpy() if hasattr(errors, "detach")
            else np.asarray(errors)).ravel()
  return int(iteration) + 1, int(inner_iterations), int(total_iter), errors


def default_progress_fn(fmt: str = "{iter} / {max_iter} -- {error}",
                        stream: Optional[io.TextIOBase] = None) -> Callable[[IOStatus], None]:
  """utils.py:105-160: prints ``fmt`` (keys ``iter``, ``max_iter``,
  ``error``) to ``stream`` (stdout by default) when the error was computed."""

  def progress_callback(status: IOStatus) -> None:
    iteration, inner, total, errors = _prepare_info(status)
    if iteration % inner == 0:
      error = errors[max(0, iteration // inner - 1)]
      print(fmt.format(iter=iteration, max_iter=total, error=error), file=stream)

  return progress_callback


def tqdm_progress_fn(pbar: Any, fmt: str = "error: {error:0.6e}") -> Callable[[IOStatus], None]:
  """utils.py:163-221: sets ``fmt`` as the bar's postfix and advances it
  when the error was computed."""

  def progress_callback(status: IOStatus) -> None:
    iteration, inner, total, errors = _prepare_info(status)
    if iteration % inner == 0:
      error = errors[max(0, iteration // inner - 1)]
      pbar.set_postfix_str(fmt.format(iter=iteration, max_iter=total, error=error))
      pbar.total = total // inner
      pbar.update()

  return progress_callback
