"""The progress callbacks (ott/utils.py:105-231) on a hand-made status."""
import io
import types

import numpy as np

from ott_b200 import utils


def _status(it, errors):
  return (it, 7, 14, types.SimpleNamespace(errors=np.asarray(errors)))


def test_default_progress_fn_prints_on_error_iterations():
  stream = io.StringIO()
  cb = utils.default_progress_fn(fmt="foo {iter}/{max_iter} {error:.3f}", stream=stream)
  cb(_status(3, [0.5, -1.0]))   # not an error iteration: nothing
  cb(_status(6, [0.5, -1.0]))   # iteration 7 of 14: block 0
  cb(_status(13, [0.5, 0.25]))  # iteration 14: block 1
  assert stream.getvalue() == "foo 7/14 0.500\nfoo 14/14 0.250\n"


def test_tqdm_progress_fn_sets_postfix_and_total():
  calls = []

  class Bar:
    total = None

    def set_postfix_str(self, s):
      calls.append(s)

    def update(self):
      calls.append("update")

  bar = Bar()
  cb = utils.tqdm_progress_fn(bar, fmt="err: {error}")
  cb(_status(6, [0.5, -1.0]))
  assert calls == ["err: 0.5", "update"] and bar.total == 2
