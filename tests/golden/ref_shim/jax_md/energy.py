"""jax_md.energy stand-in (TEST INFRASTRUCTURE ONLY).

``simple_spring(dr, length, epsilon, alpha) = epsilon / alpha * (dr - length)**alpha``
and ``simple_spring_bond`` sums it over the bond list, with dr the distance
between the bond's two atoms (jax-md's ``smap.bond`` with the metric built
from the displacement function).
"""

import numpy as _np

from jax.numpy import _wrap

from . import space


def simple_spring(dr, length=1.0, epsilon=1.0, alpha=2.0, **_):
  return epsilon / alpha * (dr - length) ** alpha


def simple_spring_bond(displacement_or_metric, bond, bond_type=None, length=1.0, epsilon=1.0,
                       alpha=2.0):
  bond = _np.asarray(bond)

  def energy_fn(r, **_):
    r = _np.asarray(r)
    if bond.shape[0] == 0:
      return _wrap(_np.zeros(()))
    dr = space.distance(displacement_or_metric(r[bond[:, 0]], r[bond[:, 1]]))
    return _wrap(_np.sum(simple_spring(dr, _np.asarray(length), _np.asarray(epsilon), alpha)))

  return energy_fn
