"""The learned initializer's float64 network oracle: hand-written gradients
against central finite differences, and Adam's bias-corrected first step."""
import numpy as np
import pytest

from oracle import mlp_np


def _params(rng, dims):
  return [(rng.standard_normal((o, i)) / np.sqrt(i), rng.standard_normal(o) * 0.1)
          for i, o in zip(dims[:-1], dims[1:])]


@pytest.mark.parametrize("weighted", [False, True])
def test_gradients_match_finite_differences(weighted):
  rng = np.random.default_rng(0)
  params = _params(rng, [6, 5, 4, 3])
  x = rng.standard_normal((7, 6))
  t = rng.standard_normal((7, 3))
  lw = rng.uniform(0.1, 2.0, size=(7, 3)) if weighted else None
  loss, grads = mlp_np.loss_and_grads(params, x, t, lw)
  h = 1e-6
  for l, (w, b) in enumerate(params):
    for arr, g in ((w, grads[l][0]), (b, grads[l][1])):
      flat = arr.reshape(-1)
      gflat = g.reshape(-1)
      for k in range(0, flat.size, 3):
        old = flat[k]
        flat[k] = old + h
        lp = mlp_np.loss_and_grads(params, x, t, lw)[0].mean()
        flat[k] = old - h
        lm = mlp_np.loss_and_grads(params, x, t, lw)[0].mean()
        flat[k] = old
        np.testing.assert_allclose(gflat[k], (lp - lm) / (2 * h), rtol=1e-5, atol=1e-9)


def test_loss_is_shift_invariant():
  rng = np.random.default_rng(1)
  params = _params(rng, [4, 5, 3])
  x = rng.standard_normal((5, 4))
  t = rng.standard_normal((5, 3))
  l0 = mlp_np.loss_and_grads(params, x, t)[0]
  l1 = mlp_np.loss_and_grads(params, x, t + 3.0 - (t + 3.0).mean(1, keepdims=True))[0]
  l2 = mlp_np.loss_and_grads(params, x, t - t.mean(1, keepdims=True))[0]
  np.testing.assert_allclose(l1, l2, rtol=1e-12)
  assert np.all(l0 >= l2 - 1e-12)


def test_adam_first_step_is_signed_lr():
  rng = np.random.default_rng(2)
  params = _params(rng, [3, 2])
  grads = [(rng.standard_normal((2, 3)), rng.standard_normal(2))]
  state = [[np.zeros((2, 3)), np.zeros((2, 3)), np.zeros(2), np.zeros(2)]]
  new = mlp_np.adam_step(params, grads, state, step=1, lr=1e-2, eps=0.0)
  np.testing.assert_allclose(new[0][0], params[0][0] - 1e-2 * np.sign(grads[0][0]))
  np.testing.assert_allclose(new[0][1], params[0][1] - 1e-2 * np.sign(grads[0][1]))


def test_bf16_rounding():
  v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
  r = mlp_np.bf16(v)
  # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
  np.testing.assert_array_equal(r[:2], [1.0, 1.0])
  assert r[2] == np.float32(1.0078125)
  assert abs(r[3] + 3.140625) < 1e-7 and r[4] == 0.0
