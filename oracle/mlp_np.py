"""Float64 NumPy restatement of the learned initializer's network (TEST
INFRASTRUCTURE ONLY): Dense layers y = x W^T + b, tanh-GELU between layers,
linear last layer (the meta model of
initializers/neural/meta_initializer.py:192-207), the centred squared-error
loss and its gradients (by hand, checked against finite differences in the
tests), and Adam (Kingma & Ba, the optax.adam update of
meta_initializer.py:77-78)."""
import numpy as np

C = np.sqrt(2.0 / np.pi)


def gelu(z):
  return 0.5 * z * (1.0 + np.tanh(C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
  t = np.tanh(C * (z + 0.044715 * z ** 3))
  return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C * (1.0 + 3 * 0.044715 * z * z)


def forward(params, x):
  """params: list of (W [out, in], b [out]). Returns y and the cache."""
  acts, zs = [x], []
  h = x
  for l, (w, b) in enumerate(params):
    z = h @ w.T + b
    zs.append(z)
    h = z if l + 1 == len(params) else gelu(z)
    acts.append(h)
  return h, (acts, zs)


def loss_and_grads(params, x, t, w=None):
  """Batch mean of the (optionally weighted) centred squared error
  sum_j w_j ((y_j - t_j) - s)^2 / sum_j w_j, s the weighted mean of y - t,
  and its gradients (the residual has zero weighted mean, so
  d loss / d y_j = 2 w_j r_j / (sum w B))."""
  y, (acts, zs) = forward(params, x)
  B, m = y.shape
  w = np.ones_like(y) if w is None else np.asarray(w, np.float64)
  sw = w.sum(axis=1, keepdims=True)
  diff = y - t
  r = diff - (w * diff).sum(axis=1, keepdims=True) / sw
  loss_per = (w * r * r).sum(axis=1) / sw[:, 0]
  dz = 2.0 * w * r / (sw * B)
  grads = [None] * len(params)
  for l in range(len(params) - 1, -1, -1):
    w_l, _ = params[l]
    grads[l] = (dz.T @ acts[l], dz.sum(axis=0))
    if l > 0:
      dz = (dz @ w_l) * gelu_grad(zs[l - 1])
  return loss_per, grads


def adam_step(params, grads, state, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
  out = []
  for (w, b), (gw, gb), st in zip(params, grads, state):
    new = []
    for k, (p, g) in enumerate(((w, gw), (b, gb))):
      m = b1 * st[2 * k] + (1 - b1) * g
      v = b2 * st[2 * k + 1] + (1 - b2) * g * g
      st[2 * k], st[2 * k + 1] = m, v
      new.append(p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps))
    out.append(tuple(new))
  return out


def bf16(x):
  """Rounds float32 values to bfloat16 (nearest, ties to even), returned as
  float32."""
  u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
  r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
  return r.astype(np.uint32).view(np.float32)


def forward_bf16(params, x):
  """The device forward's roundings: bf16 input and weights, FP32
  accumulation (here float64), pre-activation rounded to bf16, activation
  computed from it and rounded to bf16; the last layer stays FP32."""
  h = bf16(x).astype(np.float64)
  acts, zs = [h], []
  for l, (w, b) in enumerate(params):
    z = h @ bf16(w).astype(np.float64).T + b
    if l + 1 == len(params):
      zs.append(z)
      return z, (acts, zs)
    zb = bf16(z).astype(np.float64)
    zs.append(zb)
    h = bf16(gelu(zb)).astype(np.float64)
    acts.append(h)
