"""Inputs of the reference-run fixtures (``ref_fixtures.npz``), rebuilt the
same way by the fixture script and by the tests.

TEST INFRASTRUCTURE ONLY.  Every case is a seeded synthetic chain from
``prolix_b200.synth`` plus, where named, seeded improper and Urey-Bradley
terms, an explicit 1-4 exception table, or the real-protein case, whose
inputs (1A00 chain A from prolix's ``tests/physics/data/1a00.pqr``) are
stored in the fixture file itself because the GPU box has no reference
tree.
"""

from __future__ import annotations

import hashlib
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

from prolix_b200 import synth  # noqa: E402

FIXTURE = os.path.join(HERE, "ref_fixtures.npz")

# name -> (n_atoms, seed, compact, cmap, LJ/Coulomb cutoff (0: all pairs), extras)
CASES = {
    "chain166_periodic_imp": (166, 1, False, True, 0.0, "periodic"),
    "chain166_harmonic_imp": (166, 3, True, False, 0.0, "harmonic"),
    "globule600_cut9": (600, 600, True, True, 9.0, None),
    "chain166_exceptions": (166, 2, True, False, 0.0, "exceptions"),
}
PQR_CASE = "pqr1a00_chainA"
# the NL-Born + dense-GB split (generalized_born.py:706-817) on the 600-atom
# globule's inputs: Born radii from the pairs within SPLIT_CUTOFF, GB pair
# terms over all pairs
SPLIT_CASE = "globule600_nlborn"
SPLIT_BASE = "globule600_cut9"
SPLIT_CUTOFFS = tuple(10.0 + 0.001 * k for k in range(50))
SPLIT_MARGIN = 3e-5  # no pair distance within this of the cutoff (float32 rounding and FD steps stay on one side)
SPLIT_FD_H = 1e-5    # the split case's finite-difference step (2 h < SPLIT_MARGIN)


def split_cutoff(pos) -> float:
  """The first of SPLIT_CUTOFFS with no pair distance within SPLIT_MARGIN."""
  d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
  for c in SPLIT_CUTOFFS:
    if not np.any(np.abs(d - c) < SPLIT_MARGIN):
      return c
  raise ValueError("no cutoff clear of the pair distances")


def split_neighbors(pos, cutoff: float):
  """(N, K) neighbour rows of the pairs within ``cutoff`` (both directions,
  padded with N), as the reference's NL functions take them."""
  n = pos.shape[0]
  d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
  within = (d < cutoff) & ~np.eye(n, dtype=bool)
  k = int(within.sum(axis=1).max())
  rows = np.full((n, k), n, dtype=np.int32)
  for i in range(n):
    j = np.nonzero(within[i])[0]
    rows[i, :j.size] = j
  return rows
# OBC2 scale factors by element (the defaults of OpenMM's GBSAOBCForce
# parameter sets, which prolix's OpenMM parity tests compare against)
OBC_SCALE = {"H": 0.85, "C": 0.72, "N": 0.79, "O": 0.85, "S": 0.96}


def digest(*arrays) -> str:
  h = hashlib.sha256()
  for a in arrays:
    h.update(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes())
  return h.hexdigest()[:16]


def add_impropers_ub(s: dict, form: str, seed: int) -> dict:
  """Impropers (i, i+2, i+1, i+3) every 5 atoms and Urey-Bradley springs
  (i, i+2) every 3 atoms, parameters drawn from ``default_rng(seed)``.
  ``form`` "periodic": rows (M, 2, 3) = (n, phase, k) with n = 2, phase pi
  and n = 1, phase 0; "harmonic": rows (M, 1, 2) = (k, phi0) with phi0
  anywhere in (-pi, pi), so the wrap of the difference is exercised."""
  rng = np.random.default_rng(seed)
  pos = np.asarray(s["positions"], np.float64)
  n = pos.shape[0]
  start = np.arange(0, n - 3, 5)
  imp = np.stack([start, start + 2, start + 1, start + 3], axis=1).astype(np.int32)
  m = imp.shape[0]
  if form == "periodic":
    k = rng.uniform(0.5, 5.0, size=(m, 2))
    params = np.stack([np.stack([np.full(m, 2.0), np.full(m, math.pi), k[:, 0]], 1),
                       np.stack([np.full(m, 1.0), np.zeros(m), k[:, 1]], 1)], axis=1)
  elif form == "harmonic":
    params = np.stack([rng.uniform(5.0, 50.0, size=m), rng.uniform(-math.pi, math.pi, size=m)],
                      axis=1)[:, None, :]
  else:
    raise ValueError(form)
  ub0 = np.arange(0, n - 2, 3)
  ub = np.stack([ub0, ub0 + 2], axis=1).astype(np.int32)
  r = np.linalg.norm(pos[ub[:, 0]] - pos[ub[:, 1]], axis=1)
  ubp = np.stack([r + rng.uniform(-0.1, 0.1, size=r.shape[0]),
                  rng.uniform(10.0, 50.0, size=r.shape[0])], axis=1)
  return dict(s, impropers=imp, improper_params=params, urey_bradley_bonds=ub,
              urey_bradley_params=ubp)


def exception_table(s: dict):
  """(pairs_14, params (chargeprod, sigma, epsilon)) in the layout proxide
  hands ExclusionSpec.from_protein (physics/neighbor_list.py:105-125), with
  per-pair values that differ from the global 1-4 scaling."""
  from prolix_b200 import topology
  n = len(s["charges"])
  pairs, kind = topology.exclusion_pairs(s["bonds"], n)
  p14 = pairs[kind == 1].astype(np.int32)
  q = np.asarray(s["charges"], np.float64)
  sig = np.asarray(s["sigmas"], np.float64)
  eps = np.asarray(s["epsilons"], np.float64)
  i, j = p14[:, 0], p14[:, 1]
  params = np.stack([q[i] * q[j] * 0.8333333, 0.5 * (sig[i] + sig[j]) * 1.05,
                     0.5 * np.sqrt(eps[i] * eps[j])], axis=1)
  return p14, params


def case_system(name: str):
  """(system dict, LJ/Coulomb cutoff) of a synthetic case.  The generated
  positions sit exactly at the bonds' and angles' rest values, so they are
  displaced by N(0, 0.03 A) noise (``default_rng(seed + 2000)``) to give
  those terms energy and force."""
  n, seed, compact, cmap, cutoff, extra = CASES[name]
  s = synth.make_chain(n, seed, compact=compact, cmap=cmap)
  rng = np.random.default_rng(seed + 2000)
  s["positions"] = np.asarray(s["positions"], np.float64) + rng.normal(0.0, 0.03, size=(n, 3))
  if extra in ("periodic", "harmonic"):
    s = add_impropers_ub(s, extra, seed + 1000)
  return s, cutoff


def read_pqr(path: str, chain: str = "A"):
  """positions (N, 3), charges, radii and element letters of one chain."""
  pos, q, rad, elem = [], [], [], []
  with open(path) as f:
    for line in f:
      if not line.startswith(("ATOM", "HETATM")):
        continue
      parts = line.split()
      if len(parts) != 11:
        raise ValueError(f"unexpected PQR record: {line!r}")
      if parts[4] != chain:
        continue
      x, y, z, qq, rr = (float(v) for v in parts[-5:])
      pos.append((x, y, z))
      q.append(qq)
      rad.append(rr)
      elem.append(next(c for c in parts[2] if c.isalpha()))
  return np.array(pos), np.array(q), np.array(rad), elem


def pqr_scaled_radii(radii, elements):
  return np.array([r * OBC_SCALE.get(e, 0.8) for r, e in zip(radii, elements)])
