"""NumPy stand-in for the parts of ``jax`` that prolix's force-field source
files use, so that those files run unmodified in FP64 where JAX is absent.

TEST INFRASTRUCTURE ONLY (``tests/golden/make_ref_fixtures.py``).

* ``vmap``: a loop over the mapped axis with the results stacked; a function
  marked ``_elementwise`` (the free-space displacement) is instead called
  once on the broadcast arguments, which gives the same values.
* ``custom_vjp``: calls the primal function; ``defvjp`` keeps the forward
  and backward rules as attributes, so the fixture script can call the
  reference's hand-written backward rule (its analytic forces) directly.
* ``jit``, ``checkpoint``: identity.  There is no automatic differentiation.
"""

from __future__ import annotations

import functools as _ft

import numpy as _np

from . import lax, numpy, scipy  # noqa: F401
from .numpy import _wrap


class _Config:
  jax_enable_x64 = True

  def update(self, *_a, **_k):
    pass


config = _Config()
Array = _np.ndarray


def jit(fun=None, **_kw):
  if fun is None:
    return lambda f: f
  return fun


def checkpoint(fun=None, **_kw):
  if fun is None:
    return lambda f: f
  return fun


remat = checkpoint


class _Debug:
  @staticmethod
  def print(*_a, **_k):
    pass


debug = _Debug()


def _take(a, axis, i):
  a = _np.asarray(a)
  idx = (slice(None),) * axis + (i, Ellipsis)
  return _wrap(a[idx])


def _stack(outs):
  first = outs[0]
  if first is None:
    return None
  if isinstance(first, tuple) and not hasattr(first, "_fields"):
    return tuple(_stack([o[k] for o in outs]) for k in range(len(first)))
  if isinstance(first, list):
    return [_stack([o[k] for o in outs]) for k in range(len(first))]
  if isinstance(first, dict):
    return {k: _stack([o[k] for o in outs]) for k in first}
  if hasattr(first, "_fields"):
    return type(first)(*(_stack([getattr(o, f) for o in outs]) for f in first._fields))
  return _wrap(_np.stack([_np.asarray(o) for o in outs]))


def vmap(fun, in_axes=0, out_axes=0, **_kw):
  if out_axes != 0:
    raise NotImplementedError("the stand-in vmap maps outputs along axis 0 only")

  def axes_for(args):
    if isinstance(in_axes, (tuple, list)):
      if len(in_axes) != len(args):
        raise ValueError("in_axes length does not match the arguments")
      return tuple(in_axes)
    return (in_axes,) * len(args)

  if getattr(fun, "_elementwise", False):
    # (no functools.wraps: it would copy the _elementwise mark onto vec,
    # whose own mapped axis is no longer elementwise)
    def vec(*args):
      moved = []
      for a, ax in zip(args, axes_for(args)):
        a = _np.asarray(a)
        moved.append(a[None] if ax is None else _np.moveaxis(a, ax, 0))
      return _wrap(fun(*moved))
    return vec

  def looped(*args):
    axes = axes_for(args)
    sizes = {_np.asarray(a).shape[ax] for a, ax in zip(args, axes) if ax is not None}
    if len(sizes) != 1:
      raise ValueError(f"vmap: mapped axes have sizes {sizes}")
    n = sizes.pop()
    outs = [fun(*[a if ax is None else _take(a, ax, i) for a, ax in zip(args, axes)])
            for i in range(n)]
    return _stack(outs)

  return looped


class custom_vjp:  # noqa: N801  (JAX's name)
  def __init__(self, fun, nondiff_argnums=()):
    self.fun = fun
    self.nondiff_argnums = tuple(nondiff_argnums)
    self.fwd = None
    self.bwd = None
    _ft.update_wrapper(self, fun)

  def __call__(self, *args, **kwargs):
    return self.fun(*args, **kwargs)

  def defvjp(self, fwd, bwd):
    self.fwd, self.bwd = fwd, bwd


class custom_jvp(custom_vjp):  # noqa: N801
  def defjvp(self, jvp):
    self.jvp = jvp


def grad(*_a, **_k):
  raise NotImplementedError("the NumPy stand-in has no automatic differentiation")


vjp = grad
value_and_grad = grad
