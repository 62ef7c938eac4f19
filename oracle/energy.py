"""Total implicit-solvent energy and forces (bonded + nonbonded), FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Mirrors the term split of prolix ``make_energy_fn(..., implicit_solvent=True)``
(system.py:229-270): bond, angle, dihedral, cmap, lj, and electrostatics as
(GB polar, direct Coulomb) plus the ACE nonpolar term.
"""

from __future__ import annotations

import numpy as np

from . import bonded, gbsa

TERMS = ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar")


def energy_forces(system, pos, cutoff=0.0, **kw):
  """Return (energies dict incl. 'total', forces (N, 3), extras)."""
  pos = np.asarray(pos, np.float64)
  eb, fb = bonded.bonded_all(system, pos)
  en, fn, extras = gbsa.nonbonded(system, pos, cutoff, **kw)
  e = {**eb, **en}
  e["total"] = float(sum(e[t] for t in TERMS))
  return e, fb + fn, extras


def total_energy(system, pos, cutoff=0.0, **kw):
  return energy_forces(system, pos, cutoff, **kw)[0]["total"]
