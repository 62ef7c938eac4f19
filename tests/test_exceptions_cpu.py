"""Explicit 1-4 exception pairs (prolix bonded.py:186-230, ExclusionSpec
neighbor_list.py:44-142) in the oracle: moving the 1-4 pairs out of the
scaled LJ/Coulomb kernels into exception terms whose parameters carry the
same scales gives the same energies and forces."""

import numpy as np

from oracle import energy, topology
from prolix_b200 import synth


def with_explicit_14(s, sigma_jitter=0.0, seed=0):
  """The system with its 1-4 pairs excluded (kind 0) and restated as
  exception pairs, parameters pre-scaled as ExclusionSpec.from_protein
  expects them."""
  n = len(s["charges"])
  p12, p13, p14 = topology.bonded_pairs(s["bonds"], n)
  allp = np.concatenate([p12, p13, p14]).astype(np.int64)
  allp = np.sort(allp, axis=1)
  allp = allp[np.lexsort((allp[:, 1], allp[:, 0]))]
  q, sig, eps = (np.asarray(s[k], np.float64) for k in ("charges", "sigmas", "epsilons"))
  i, j = p14[:, 0], p14[:, 1]
  sij = 0.5 * (sig[i] + sig[j])
  if sigma_jitter:
    sij = sij * np.random.default_rng(seed).uniform(1 - sigma_jitter, 1 + sigma_jitter, len(i))
  return dict(s, excl_pairs=allp.astype(np.int32), excl_kind=np.zeros(len(allp), np.int32),
              exception_pairs=p14.astype(np.int32),
              exception_chargeprods=q[i] * q[j] * topology.COUL14_SCALE,
              exception_sigmas=sij,
              exception_epsilons=topology.LJ14_SCALE * np.sqrt(eps[i] * eps[j]))


def test_explicit_14_pairs_equal_the_scaled_ones():
  s = synth.make_chain(80, 3, compact=True)
  e0, f0, _ = energy.energy_forces(s, s["positions"])
  ex = with_explicit_14(s)
  e1, f1, _ = energy.energy_forces(ex, ex["positions"])
  assert e0["exception"] == 0.0 and e1["exception"] != 0.0
  for t in ("bond", "angle", "dihedral", "gb", "nonpolar"):
    assert e1[t] == e0[t], t
  a = e0["lj"] + e0["coulomb"]
  b = e1["lj"] + e1["coulomb"] + e1["exception"]
  assert abs(a - b) <= 1e-9 * abs(a)
  assert abs(e1["total"] - e0["total"]) <= 1e-9 * abs(e0["total"])
  np.testing.assert_allclose(f1, f0, rtol=0, atol=1e-9 * np.abs(f0).max())
