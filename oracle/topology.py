"""Exclusion topology (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates prolix's 1-2 / 1-3 / 1-4 rule and its per-pair scale table:

* ``find_bonded_exclusions`` utils/topology.py:26-93: breadth-first walk of
  the bond graph to depth three; a pair keeps its shortest separation
  (1-3 minus 1-2, 1-4 minus 1-2 and 1-3).
* ``ExclusionSpec.from_protein`` physics/neighbor_list.py:52-142 and
  ``map_exclusions_to_dense_padded`` :236-303: 1-2 and 1-3 pairs get scale 0
  for both LJ and Coulomb; 1-4 pairs get (vdw 0.5, elec 0.83333333), stored
  as float32 in the reference's table, hence the float32 rounding below.
"""

from __future__ import annotations

import collections

import numpy as np

LJ14_SCALE = float(np.float32(0.5))
COUL14_SCALE = float(np.float32(0.83333333))


def bonded_pairs(bonds: np.ndarray, n_atoms: int):
  """Return (pairs12, pairs13, pairs14) as sorted (M, 2) int arrays with i < j."""
  adj = collections.defaultdict(list)
  for a, b in np.asarray(bonds, dtype=np.int64).reshape(-1, 2):
    adj[int(a)].append(int(b))
    adj[int(b)].append(int(a))
  s12, s13, s14 = set(), set(), set()
  for i in range(n_atoms):
    for j in adj[i]:
      if j > i:
        s12.add((i, j))
      for k in adj[j]:
        if k == i:
          continue
        if k > i:
          s13.add((i, k))
        for l in adj[k]:
          if l in (j, i):
            continue
          if l > i:
            s14.add((i, l))
  s13 -= s12
  s14 = (s14 - s12) - s13

  def arr(s):
    return np.array(sorted(s), dtype=np.int64).reshape(-1, 2)

  return arr(s12), arr(s13), arr(s14)


def pair_scales(bonds, n_atoms, lj14=LJ14_SCALE, coul14=COUL14_SCALE):
  """Sparse scale table: list of (i, j, s_vdw, s_elec) for i < j, sorted."""
  p12, p13, p14 = bonded_pairs(bonds, n_atoms)
  rows = []
  for i, j in np.concatenate([p12, p13]):
    rows.append((int(i), int(j), 0.0, 0.0))
  for i, j in p14:
    rows.append((int(i), int(j), lj14, coul14))
  rows.sort()
  if not rows:
    return np.zeros((0, 2), np.int64), np.zeros(0), np.zeros(0)
  a = np.array(rows)
  return a[:, :2].astype(np.int64), a[:, 2].copy(), a[:, 3].copy()
