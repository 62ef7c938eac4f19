"""Total implicit-solvent energy and forces (bonded + nonbonded), FP64.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Mirrors the term split of prolix ``make_energy_fn(..., implicit_solvent=True)``
(system.py:229-270): bond, angle, dihedral, improper, Urey-Bradley, cmap, lj,
and electrostatics as
(GB polar, direct Coulomb) plus the ACE nonpolar term and the explicit 1-4
exception pairs.
"""

from __future__ import annotations

import numpy as np

from . import bonded, gbsa

TERMS = ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar", "exception",
         "improper", "urey_bradley")


def energy_forces(system, pos, cutoff=0.0, **kw):
  """Return (energies dict incl. 'total', forces (N, 3), extras).  The
  ``exception`` term is the explicit 1-4 pair list of an ExclusionSpec
  (system keys ``exception_pairs``, ``exception_sigmas``,
  ``exception_epsilons``, ``exception_chargeprods``; system.py:149-159); its
  pairs are excluded from LJ/Coulomb through the system's exclusion list."""
  pos = np.asarray(pos, np.float64)
  eb, fb = bonded.bonded_all(system, pos)
  en, fn, extras = gbsa.nonbonded(system, pos, cutoff, **kw)
  ex, fx = bonded.exception_pairs(pos, system.get("exception_pairs", np.zeros((0, 2))),
                                  system.get("exception_sigmas", np.zeros(0)),
                                  system.get("exception_epsilons", np.zeros(0)),
                                  system.get("exception_chargeprods", np.zeros(0)),
                                  kw.get("k_coul", gbsa.K_COULOMB))
  e = {**eb, **en, "exception": ex}
  e["total"] = float(sum(e[t] for t in TERMS))
  return e, fb + fn + fx, extras


def total_energy(system, pos, cutoff=0.0, **kw):
  return energy_forces(system, pos, cutoff, **kw)[0]["total"]
