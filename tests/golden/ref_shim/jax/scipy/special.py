"""Stand-in for ``jax.scipy.special`` on SciPy (TEST INFRASTRUCTURE ONLY)."""

import scipy.special as _sp

from ..numpy import _wrap


def erf(x):
  return _wrap(_sp.erf(x))


def erfc(x):
  return _wrap(_sp.erfc(x))
