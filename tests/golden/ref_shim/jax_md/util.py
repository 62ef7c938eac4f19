"""jax_md.util stand-in (TEST INFRASTRUCTURE ONLY)."""

import numpy as _np

Array = _np.ndarray
f32 = _np.float64
f64 = _np.float64
i32 = _np.int32


def high_precision_sum(x, axis=None, keepdims=False):
  return _np.sum(_np.asarray(x, _np.float64), axis=axis, keepdims=keepdims)
