"""The C/OpenMP oracle agrees with the NumPy oracle (CPU only)."""

import numpy as np
import pytest

from oracle import bonded, cforces, gbsa
from prolix_b200 import synth


@pytest.mark.parametrize("cutoff,gb_cutoff", [(0.0, None), (9.0, None), (9.0, 0.0), (7.0, 11.0)])
def test_c_oracle_matches_numpy_oracle(cutoff, gb_cutoff):
  s = synth.make_chain(350, 21, compact=True)
  pos = s["positions"] + np.random.default_rng(3).normal(0, 0.05, size=s["positions"].shape)
  ec, fc = cforces.energy_forces(s, pos, cutoff=cutoff, gb_cutoff=gb_cutoff, threads=2)
  eb, fb = bonded.bonded_all(s, pos)
  en, fn, _ = gbsa.nonbonded(s, pos, cutoff, gb_cutoff=gb_cutoff)
  ref = {**eb, **en}
  for k in ("bond", "angle", "dihedral", "lj", "coulomb", "gb", "nonpolar"):
    assert ec[k] == pytest.approx(ref[k], rel=1e-11, abs=1e-9), k
  np.testing.assert_allclose(fc, fb + fn - bonded.cmap(pos, np.zeros((0, 5)), [], [])[1],
                             rtol=1e-10, atol=1e-9)
