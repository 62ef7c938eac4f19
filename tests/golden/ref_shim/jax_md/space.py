"""jax_md.space stand-in (TEST INFRASTRUCTURE ONLY).

``free()`` is jax-md's free-space pair (displacement Ra - Rb, shift R + dR);
``distance`` is the Euclidean norm over the last axis (0 where it is 0).
"""

import numpy as _np

from jax.numpy import _wrap

DisplacementFn = object
ShiftFn = object


def _displacement(ra, rb, **_):
  return _wrap(_np.asarray(ra) - _np.asarray(rb))


_displacement._elementwise = True


def _shift(r, dr, **_):
  return _wrap(_np.asarray(r) + _np.asarray(dr))


def free():
  return _displacement, _shift


def square_distance(dr):
  return _wrap(_np.sum(_np.asarray(dr) ** 2, axis=-1))


def distance(dr):
  d2 = square_distance(dr)
  return _wrap(_np.where(d2 > 0, _np.sqrt(_np.where(d2 > 0, d2, 1.0)), 0.0))


def map_bond(metric_or_displacement):
  def fn(ra, rb, **kw):
    return metric_or_displacement(ra, rb, **kw)
  return fn
