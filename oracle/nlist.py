"""Neighbour lists by brute force (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

jax_md's ``partition.neighbor_list`` as prolix configures it
(physics/neighbor_list.py:155-172, batched_simulate.py:1429-1464): atom j is
a neighbour of i (j != i) when |r_i - r_j| < cutoff + dr_threshold (the
skin); the list holds both (i, j) and (j, i); it is rebuilt when some atom
moved more than dr_threshold / 2 since the last build
(batched_simulate.py:1600-1622).
"""

from __future__ import annotations

import numpy as np


def neighbour_sets(pos, reach):
  """List of sets: neighbours of each atom within ``reach``."""
  pos = np.asarray(pos, dtype=np.float64)
  n = pos.shape[0]
  out = []
  for a in range(0, n, 512):
    d = pos[a:a + 512, None, :] - pos[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", d, d)
    for k in range(r2.shape[0]):
      hits = np.nonzero(r2[k] < reach * reach)[0]
      out.append(set(int(j) for j in hits if j != a + k))
  return out


def needs_rebuild(pos, pos_ref, skin):
  d = np.asarray(pos) - np.asarray(pos_ref)
  return bool(np.max(np.einsum("ij,ij->i", d, d)) > (0.5 * skin) ** 2)
