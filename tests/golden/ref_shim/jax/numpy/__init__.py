"""NumPy stand-in for ``jax.numpy``, in FP64.

TEST INFRASTRUCTURE ONLY: lets ``tests/golden/make_ref_fixtures.py`` run
prolix's own source files where JAX is not installed.  Every function
forwards to NumPy; arrays carry JAX's functional ``.at[...]`` update
interface; float32 requests become float64, so the reference's arithmetic
runs in double precision throughout (the precision the fixtures are quoted
in).  Only what the loaded reference modules use is provided.
"""

from __future__ import annotations

import numpy as _np


class Array(_np.ndarray):
  """ndarray with JAX's ``x.at[idx].set / add / multiply / get``."""

  @property
  def at(self):
    return _At(self)


class _At:
  def __init__(self, arr):
    self._arr = arr

  def __getitem__(self, idx):
    return _AtIndex(self._arr, idx)


class _AtIndex:
  def __init__(self, arr, idx):
    self._arr, self._idx = arr, _unwrap_index(idx)

  def set(self, v):
    out = _np.array(self._arr, copy=True)
    out[self._idx] = _np.asarray(v)
    return _wrap(out)

  def add(self, v):
    out = _np.array(self._arr, copy=True)
    _np.add.at(out, self._idx, _np.asarray(v))
    return _wrap(out)

  def multiply(self, v):
    out = _np.array(self._arr, copy=True)
    _np.multiply.at(out, self._idx, _np.asarray(v))
    return _wrap(out)

  def get(self, **_):
    return _wrap(_np.asarray(self._arr)[self._idx])


def _unwrap_index(idx):
  if isinstance(idx, tuple):
    return tuple(_unwrap_index(i) for i in idx)
  if isinstance(idx, _np.ndarray):
    return _np.asarray(idx)
  return idx


def _fix_dtype(dt):
  if dt is None:
    return None
  d = _np.dtype(dt)
  if d == _np.float32 or d == _np.float16:
    return _np.float64
  return dt


def _wrap(x):
  if isinstance(x, _np.ndarray):
    if x.dtype == _np.float32:
      x = x.astype(_np.float64)
    return x if isinstance(x, Array) else x.view(Array)
  if isinstance(x, tuple):
    return type(x)(_wrap(v) for v in x) if not hasattr(x, "_fields") else x
  return x


def _forward(fn):
  def call(*args, **kwargs):
    if "dtype" in kwargs:
      kwargs["dtype"] = _fix_dtype(kwargs["dtype"])
    return _wrap(fn(*args, **kwargs))
  call.__name__ = getattr(fn, "__name__", "fn")
  return call


def array(obj, dtype=None, copy=True, **_):
  a = _np.array(obj, dtype=_fix_dtype(dtype), copy=copy)
  return _wrap(a)


def asarray(obj, dtype=None, **_):
  return _wrap(_np.asarray(obj, dtype=_fix_dtype(dtype)))


ndarray = _np.ndarray
float64 = _np.float64
float32 = _np.float64  # FP64 throughout
float16 = _np.float64
int32 = _np.int32
int64 = _np.int64
uint32 = _np.uint32
bool_ = _np.bool_
pi = _np.pi
inf = _np.inf
nan = _np.nan
newaxis = None
e = _np.e


class _Linalg:
  def __getattr__(self, name):
    return _forward(getattr(_np.linalg, name))


linalg = _Linalg()


def __getattr__(name):
  fn = getattr(_np, name)
  if callable(fn) and not isinstance(fn, type):
    return _forward(fn)
  return fn
