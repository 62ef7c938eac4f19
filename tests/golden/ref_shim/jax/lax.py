"""NumPy stand-in for the ``jax.lax`` control flow and slicing prolix uses.

TEST INFRASTRUCTURE ONLY.  ``dynamic_slice`` clamps its start indices into
range as XLA does; ``scan`` runs its body in a Python loop.
"""

from __future__ import annotations

import numpy as _np

from .numpy import _wrap


def dynamic_slice(operand, start_indices, slice_sizes):
  a = _np.asarray(operand)
  idx = []
  for dim, (s, n) in enumerate(zip(start_indices, slice_sizes)):
    s = int(s)
    s = min(max(s, 0), a.shape[dim] - int(n))
    idx.append(slice(s, s + int(n)))
  return _wrap(a[tuple(idx)])


def dynamic_update_slice(operand, update, start_indices):
  a = _np.array(operand, copy=True)
  u = _np.asarray(update)
  idx = []
  for dim, s in enumerate(start_indices):
    s = min(max(int(s), 0), a.shape[dim] - u.shape[dim])
    idx.append(slice(s, s + u.shape[dim]))
  a[tuple(idx)] = u
  return _wrap(a)


def scan(f, init, xs=None, length=None, **_kw):
  from . import _stack
  if xs is None:
    items = [None] * int(length)
  else:
    items = [x for x in _np.asarray(xs)] if not isinstance(xs, (tuple, list)) else \
        list(zip(*[_np.asarray(x) for x in xs]))
  carry, ys = init, []
  for x in items:
    carry, y = f(carry, _wrap(x) if isinstance(x, _np.ndarray) else x)
    ys.append(y)
  if not ys or all(y is None for y in ys):
    return carry, None
  return carry, _stack(ys)


def fori_loop(lower, upper, body, init):
  v = init
  for i in range(int(lower), int(upper)):
    v = body(i, v)
  return v


def cond(pred, true_fun, false_fun, *operands):
  return true_fun(*operands) if bool(pred) else false_fun(*operands)


def select(pred, on_true, on_false):
  return _wrap(_np.where(pred, on_true, on_false))


def stop_gradient(x):
  return x
