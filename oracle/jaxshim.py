"""A NumPy stand-in for the part of the jax API that ott-jax's Sinkhorn path
calls (TEST INFRASTRUCTURE ONLY).

jax is not installed in this image. To pin the oracle against the
reference's own source, ``oracle/reference_loader.py`` executes the
reference's Python files for the path (geometry, costs, pointcloud, linear
problem, initializers, fixed-point loop, Sinkhorn, solve) with ``jax`` bound
to this module. Every array function maps to its NumPy equivalent with the
same semantics; control flow (``lax.while_loop``, ``lax.scan``,
``lax.cond``) runs as Python loops; ``vmap`` loops over the mapped axis;
transformations that only matter for differentiation (``custom_jvp``,
``custom_vjp``, ``stop_gradient``, pytree registration, ``jit``) are
identities. ``jax.scipy.special.logsumexp`` is the published max-shifted
algorithm as restated in ``oracle/sinkhorn_np.py``.

``install(x64=True)`` keeps NumPy dtypes (float64 inputs reproduce the
reference under ``jax_enable_x64``); ``install(x64=False)`` narrows every
float64 result to float32, as jax does with 64-bit types disabled.
"""
from __future__ import annotations

import functools
import sys
import types
from typing import Any, Callable

import numpy as np


class JArray(np.ndarray):
  """ndarray with jax's functional ``.at[idx].set(v)`` update."""

  def repeat(self, repeats, axis=None, total_repeat_length=None):
    """jnp.ndarray.repeat: ``total_repeat_length`` fixes the output length
    (truncated, or padded with the last element)."""
    out = np.repeat(np.asarray(self), np.asarray(repeats), axis=axis)
    if total_repeat_length is not None:
      n = int(total_repeat_length)
      out = out[:n] if len(out) >= n else np.concatenate([out, np.repeat(out[-1:], n - len(out))])
    return wrap(out)

  @property
  def at(self):
    arr = self

    class _Indexer:
      def __getitem__(self, idx):
        class _Upd:
          def set(self, v):
            out = np.array(arr, copy=True).view(JArray)
            out[idx] = v
            return out

          def add(self, v):
            out = np.array(arr, copy=True).view(JArray)
            out[idx] += v
            return out

          def get(self):
            # jax clamps out-of-bounds gather indices to the array bounds
            if isinstance(idx, np.ndarray) and idx.dtype.kind in "iu":
              return wrap(arr[np.clip(idx, 0, arr.shape[0] - 1)])
            return wrap(arr[idx])
        return _Upd()
    return _Indexer()


# False mimics jax with jax_enable_x64 off: no 64-bit floats exist.
X64 = True


def _narrow(x):
  if not X64 and isinstance(x, np.ndarray) and x.dtype == np.float64:
    return x.astype(np.float32)
  return x


def wrap(x):
  if isinstance(x, np.ndarray):
    x = _narrow(x)
    return x if isinstance(x, JArray) else x.view(JArray)
  if isinstance(x, (np.generic, float)) and not isinstance(x, (bool, np.bool_)):
    if isinstance(x, float) and X64:
      return x
    return _narrow(np.asarray(x)).view(JArray)
  if isinstance(x, tuple):
    return tuple(wrap(v) for v in x)
  if isinstance(x, list):
    return [wrap(v) for v in x]
  return x


def _wrapped(fn):
  @functools.wraps(fn)
  def f(*args, **kwargs):
    return wrap(fn(*args, **kwargs))
  return f


# ---------------------------------------------------------------- jax.numpy
def _make_jnp() -> types.ModuleType:
  m = types.ModuleType("jax.numpy")

  def __getattr__(name):
    attr = getattr(np, name)
    if callable(attr) and not isinstance(attr, type):
      return _wrapped(attr)
    return attr

  m.__getattr__ = __getattr__
  m.ndarray = np.ndarray
  m.newaxis = None
  m.inf = np.inf
  m.nan = np.nan
  m.pi = np.pi
  m.e = np.e
  m.float32 = np.float32
  m.float64 = np.float64
  m.float16 = np.float16
  m.int32 = np.int32
  m.int64 = np.int64
  m.bool_ = np.bool_
  m.dtype = np.dtype
  m.finfo = np.finfo
  m.linalg = np.linalg

  def asarray(x, dtype=None):
    return wrap(np.asarray(x, dtype=dtype))
  m.asarray = asarray
  m.array = lambda x, dtype=None, copy=True: wrap(np.array(x, dtype=dtype, copy=copy))

  def vdot(a, b):
    return wrap(np.vdot(np.asarray(a), np.asarray(b)))
  m.vdot = vdot
  return m


# ---------------------------------------------------------------- jax.lax
def _make_lax() -> types.ModuleType:
  m = types.ModuleType("jax.lax")

  def dynamic_slice(operand, start_indices, slice_sizes):
    """lax.dynamic_slice: starts clamped so that the slice fits."""
    a = np.asarray(operand)
    idx = []
    for dim, (st, sz) in enumerate(zip(start_indices, slice_sizes)):
      st = int(min(max(int(st), 0), a.shape[dim] - int(sz)))
      idx.append(slice(st, st + int(sz)))
    return wrap(a[tuple(idx)])

  m.dynamic_slice = dynamic_slice

  def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
      val = body_fun(val)
    return val

  def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    if xs is None:
      n = int(length)
      items = [None] * n
    else:
      n = len(xs)
      items = [xs[i] for i in range(n)]
    carry, ys = init, []
    for x in items:
      carry, y = f(carry, x)
      ys.append(y)
    if all(y is None for y in ys):
      return carry, None
    return carry, wrap(np.stack([np.asarray(y) for y in ys]))

  def cond(pred, true_fun, false_fun, *operands):
    return true_fun(*operands) if bool(pred) else false_fun(*operands)

  def fori_loop(lower, upper, body_fun, init_val):
    val = init_val
    for i in range(int(lower), int(upper)):
      val = body_fun(i, val)
    return val

  m.while_loop = while_loop
  m.scan = scan
  m.cond = cond
  m.fori_loop = fori_loop
  m.stop_gradient = lambda x: x
  m.select = lambda p, a, b: wrap(np.where(p, a, b))
  m.full_like = lambda x, v: wrap(np.full_like(x, v))
  return m


# ---------------------------------------------------------------- jax.scipy
def _make_special() -> types.ModuleType:
  from oracle import sinkhorn_np

  m = types.ModuleType("jax.scipy.special")

  def logsumexp(a, axis=None, b=None, keepdims=False, return_sign=False, where=None):
    out = sinkhorn_np.logsumexp(np.asarray(a), axis=axis, b=b, return_sign=return_sign)
    if keepdims and axis is not None:
      if return_sign:
        out = (np.expand_dims(out[0], axis), np.expand_dims(out[1], axis))
      else:
        out = np.expand_dims(out, axis)
    return wrap(out)

  m.logsumexp = logsumexp
  m.entr = lambda x: wrap(sinkhorn_np.entr(np.asarray(x)))
  m.xlogy = lambda x, y: wrap(np.where(np.asarray(x) == 0, 0.0, np.asarray(x) * np.log(y)))
  return m


# ---------------------------------------------------------------- transforms
class _CustomDiff:
  """custom_jvp / custom_vjp stand-in: calls the primal function."""

  def __init__(self, fun, nondiff_argnums=()):
    self.fun = fun
    functools.update_wrapper(self, fun)

  def defjvp(self, jvp):
    return jvp

  def defvjp(self, fwd, bwd):
    return None

  def __call__(self, *args, **kwargs):
    return self.fun(*args, **kwargs)

  def __get__(self, obj, objtype=None):
    if obj is None:
      return self
    return functools.partial(self.__call__, obj)


def custom_jvp(fun=None, nondiff_argnums=()):
  if fun is None:
    return lambda f: _CustomDiff(f, nondiff_argnums)
  return _CustomDiff(fun, nondiff_argnums)


custom_vjp = custom_jvp


def vmap(fun: Callable, in_axes: Any = 0, out_axes: Any = 0) -> Callable:
  """Loops fun over the mapped axis and stacks the results (out_axes 0)."""

  def mapped(*args):
    axes = in_axes
    if not isinstance(axes, (list, tuple)):
      axes = [axes] * len(args)
    sizes = {np.shape(a)[ax] for a, ax in zip(args, axes) if ax is not None}
    assert len(sizes) == 1, sizes
    n = sizes.pop()
    outs = []
    for i in range(n):
      sl = [a if ax is None else np.take(np.asarray(a), i, axis=ax) for a, ax in zip(args, axes)]
      outs.append(fun(*[wrap(s) for s in sl]))
    if isinstance(outs[0], tuple):
      return tuple(wrap(np.stack([np.asarray(o[k]) for o in outs])) for k in range(len(outs[0])))
    return wrap(np.stack([np.asarray(o) for o in outs]))

  return mapped


def _complex_step_grad(fun: Callable, **kwargs) -> Callable:
  """``jax.grad`` of a real-analytic scalar function of one scalar (the
  only use on the path: ``jax.vmap(jax.grad(precond_fun))`` in
  implicit_differentiation.py): the complex-step derivative
  ``Im(fun(x + i h)) / h``, exact to rounding for analytic functions."""
  h = 1e-30

  def d(x):
    v = np.asarray(fun(np.asarray(x, dtype=np.complex128) + 1j * h))
    return wrap(np.asarray(np.imag(v) / h, dtype=np.asarray(x).dtype))

  return d


def install(x64: bool = True) -> types.ModuleType:
  """Registers the stand-in as ``jax`` (and its submodules) in sys.modules.
  x64=False narrows every float64 result to float32, as jax does with
  jax_enable_x64 off."""
  global X64
  X64 = x64
  jax = types.ModuleType("jax")
  jnp = _make_jnp()
  lax = _make_lax()
  special = _make_special()
  scipy = types.ModuleType("jax.scipy")
  scipy.special = special
  tree_util = types.ModuleType("jax.tree_util")
  tree_util.register_pytree_node_class = lambda cls: cls
  tree_util.register_pytree_node = lambda *a, **k: None
  tree_util.tree_map = lambda f, *trees, **k: f(*trees)
  tree_util.tree_flatten = lambda t, **k: ([t], None)
  tree = types.ModuleType("jax.tree")
  tree.map = tree_util.tree_map
  tree.flatten = tree_util.tree_flatten
  tree.leaves = lambda t, **k: [t]
  random = types.ModuleType("jax.random")
  random.key = lambda seed: np.array([0, int(seed)], dtype=np.uint32)
  random.PRNGKey = random.key
  random.split = lambda key, num=2: [key for _ in range(num)]
  debug = types.ModuleType("jax.debug")
  debug.callback = lambda f, *a, **k: f(*a, **k)
  interpreters = types.ModuleType("jax.interpreters")
  batching = types.ModuleType("jax.interpreters.batching")
  batching.is_vmappable = lambda x: False
  interpreters.batching = batching
  ops = types.ModuleType("jax.ops")

  def segment_sum(data, segment_ids, num_segments=None, indices_are_sorted=False, **k):
    data, ids = np.asarray(data), np.asarray(segment_ids)
    n = int(num_segments) if num_segments is not None else int(ids.max()) + 1
    out = np.zeros((n,) + data.shape[1:], dtype=data.dtype)
    ok = (ids >= 0) & (ids < n)
    np.add.at(out, ids[ok], data[ok])
    return wrap(out)

  ops.segment_sum = segment_sum
  nn = types.ModuleType("jax.nn")
  nn.relu = lambda x: wrap(np.maximum(x, 0))
  config = types.SimpleNamespace(update=lambda *a, **k: None)
  jax.numpy = jnp
  jax.lax = lax
  jax.scipy = scipy
  jax.tree_util = tree_util
  jax.tree = tree
  jax.random = random
  jax.debug = debug
  jax.interpreters = interpreters
  jax.nn = nn
  jax.ops = ops
  jax.config = config
  jax.Array = np.ndarray
  jax.vmap = vmap
  jax.jit = lambda f=None, **k: (f if f is not None else (lambda g: g))
  jax.custom_jvp = custom_jvp
  jax.custom_vjp = custom_vjp
  jax.grad = _complex_step_grad
  jax.value_and_grad = lambda f, **k: None
  for name, mod in {"jax": jax, "jax.numpy": jnp, "jax.lax": lax, "jax.scipy": scipy,
                    "jax.scipy.special": special, "jax.tree_util": tree_util,
                    "jax.tree": tree, "jax.random": random, "jax.debug": debug,
                    "jax.interpreters": interpreters,
                    "jax.interpreters.batching": batching, "jax.nn": nn,
                    "jax.ops": ops}.items():
    sys.modules[name] = mod
  return jax
