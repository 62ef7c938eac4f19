"""Host-side topology preparation: exclusion classes and CMAP patch
coefficients.

* Exclusions follow prolix's rule (utils/topology.py:26-93,
  physics/neighbor_list.py:52-142): pairs one, two or three bonds apart,
  each at its shortest separation; 1-2 and 1-3 pairs are excluded from
  Coulomb and LJ, 1-4 pairs are scaled.  Computed here from the bond
  adjacency by vectorised walks: pairs of neighbours of one atom are the
  two-bond candidates, pairs across the ends of one bond the three-bond
  candidates, each kept only where no shorter separation exists.
* CMAP coefficients follow prolix physics/cmap.py:166-286: periodic cubic
  spline derivatives at the grid points (d/dphi, d/dpsi, and d/dphi of
  d/dpsi), then one bicubic per patch matching values and
  spacing-scaled derivatives at its corners.  The spline second
  derivatives are obtained by diagonalising the circulant spline system
  with an FFT, and the patch polynomial from the cubic Hermite basis,
  c = A F A^T.
"""

from __future__ import annotations

import math

import numpy as np

LJ14_DEFAULT = float(np.float32(0.5))
COUL14_DEFAULT = float(np.float32(0.83333333))


def _uniq(x):
  """Sorted unique values (sort-based; faster here than np.unique's hashing)."""
  x = np.sort(x)
  if x.size:
    x = x[np.concatenate([[True], x[1:] != x[:-1]])]
  return x


def _minus(a, b):
  """Sorted unique a without the values of sorted unique b."""
  if not b.size or not a.size:
    return a
  pos = np.minimum(np.searchsorted(b, a), b.size - 1)
  return a[b[pos] != a]


def exclusion_pairs(bonds, n_atoms: int):
  """(pairs (M, 2) int32 with i < j, kind (M,) int32: 0 = 1-2/1-3, 1 = 1-4)."""
  bonds = np.asarray(bonds, dtype=np.int64).reshape(-1, 2)
  if bonds.size and (bonds.min() < 0 or bonds.max() >= n_atoms):
    raise ValueError(f"bond index out of range for {n_atoms} atoms")
  bonds = bonds[bonds[:, 0] != bonds[:, 1]]
  if bonds.shape[0] == 0 or n_atoms < 2:
    return np.zeros((0, 2), np.int32), np.zeros(0, np.int32)
  n = int(n_atoms)
  # adjacency in CSR form (both directions, duplicates removed)
  key = _uniq(np.concatenate([bonds[:, 0] * n + bonds[:, 1], bonds[:, 1] * n + bonds[:, 0]]))
  src, dst = key // n, key % n
  start = np.searchsorted(src, np.arange(n + 1))
  deg = np.diff(start)
  maxdeg = int(deg.max())

  def pair_keys(i, j):
    keep = i != j
    i, j = i[keep], j[keep]
    return _uniq(np.minimum(i, j) * n + np.maximum(i, j))

  k12 = pair_keys(src, dst)
  # two bonds: neighbours k < l of a common atom c
  cand13 = []
  for k in range(maxdeg):
    for l in range(k + 1, maxdeg):
      c = np.nonzero(deg > l)[0]
      cand13.append(pair_keys(dst[start[c] + k], dst[start[c] + l]))
  k13 = _minus(_uniq(np.concatenate(cand13)) if cand13 else np.zeros(0, np.int64), k12)
  # three bonds: a - b - c - d over every bond (b, c), a in N(b), d in N(c)
  cand14 = []
  for k in range(maxdeg):
    for l in range(maxdeg):
      e = np.nonzero((deg[src] > k) & (deg[dst] > l))[0]
      cand14.append(pair_keys(dst[start[src[e]] + k], dst[start[dst[e]] + l]))
  k12_13 = np.sort(np.concatenate([k12, k13]))
  k14 = _minus(_uniq(np.concatenate(cand14)), k12_13)
  keys = np.concatenate([k12_13, k14])
  kind = np.concatenate([np.zeros(len(k12) + len(k13), np.int32), np.ones(len(k14), np.int32)])
  order = np.argsort(keys, kind="stable")
  keys, kind = keys[order], kind[order]
  pairs = np.stack([keys // n, keys % n], axis=1).astype(np.int32)
  return pairs, kind


def pairs_from_padded_table(excl_indices, scales_vdw, scales_elec):
  """(pairs, kind, lj14, coul14) from prolix's per-atom padded exclusion
  table (``excl_indices`` (N, K) int, -1 padding; ``excl_scales_vdw`` /
  ``excl_scales_elec`` (N, K); physics/neighbor_list.py:236-303).

  The reference scales pair (i, j) by the entry for j in row i
  (optimization.py:51-53).  The batch holds two classes: excluded (both
  scales 0) and one 1-4 class with a common (vdw, elec) pair.  Entries with
  both scales 1 change nothing and are dropped.  A table with other
  scales, a j listed twice in a row (the reference would add the scales),
  or rows that disagree with each other on a pair raises ``ValueError``.
  """
  idx = np.asarray(excl_indices, dtype=np.int64)
  if idx.ndim != 2:
    raise ValueError(f"excl_indices must be (N, K), got shape {idx.shape}")
  n = idx.shape[0]
  sv = np.broadcast_to(np.asarray(scales_vdw if scales_vdw is not None else np.zeros(idx.shape),
                                  dtype=np.float64), idx.shape)
  se = np.broadcast_to(np.asarray(scales_elec if scales_elec is not None else np.zeros(idx.shape),
                                  dtype=np.float64), idx.shape)
  rows, cols = np.nonzero(idx >= 0)
  j = idx[rows, cols]
  if j.size and j.max() >= n:
    raise ValueError(f"excl_indices holds atom {int(j.max())} of a {n}-atom system")
  v, e = sv[rows, cols], se[rows, cols]
  keep = (j != rows) & ~((v == 1.0) & (e == 1.0))
  rows, j, v, e = rows[keep], j[keep], v[keep], e[keep]
  if rows.size:
    fwd = np.sort(rows * n + j)
    if np.any(fwd[1:] == fwd[:-1]):
      raise ValueError("excl_indices lists an atom twice in one row (the reference would add "
                       "the two scales); merge the entries")
    if not np.array_equal(fwd, np.sort(j * n + rows)):
      raise ValueError("excl_indices is not symmetric: a pair listed in row i must be listed "
                       "in row j too (the reference scales each direction by its own row)")
  excl = (v == 0.0) & (e == 0.0)
  scaled = np.unique(np.stack([v[~excl], e[~excl]], axis=1), axis=0)
  if scaled.shape[0] > 1:
    raise ValueError(f"excl_scales hold {scaled.shape[0]} distinct (vdw, elec) 1-4 scale pairs; "
                     "one class is supported")
  lj14, c14 = (float(scaled[0, 0]), float(scaled[0, 1])) if scaled.shape[0] else \
      (LJ14_DEFAULT, COUL14_DEFAULT)
  a, b = np.minimum(rows, j), np.maximum(rows, j)
  kind = np.where(excl, 0, 1)
  key = a * n + b
  order = np.lexsort((kind, key))
  key, kind = key[order], kind[order]
  first = np.concatenate([[True], key[1:] != key[:-1]]) if key.size else np.zeros(0, bool)
  # both directions must agree on a pair's class
  uk, inv = np.unique(key, return_inverse=True)
  kmin = np.full(uk.size, 2)
  kmax = np.full(uk.size, -1)
  np.minimum.at(kmin, inv, kind)
  np.maximum.at(kmax, inv, kind)
  if np.any(kmin != kmax):
    raise ValueError("excl_indices rows disagree on the scale of a pair")
  key, kind = key[first], kind[first]
  pairs = np.stack([key // n, key % n], axis=1).astype(np.int32).reshape(-1, 2)
  return pairs, kind.astype(np.int32), lj14, c14


def _periodic_spline_slopes(y: np.ndarray) -> np.ndarray:
  """First derivatives at the knots of the periodic cubic spline through y
  (uniform spacing h = 2 pi / n)."""
  n = y.shape[0]
  h = 2.0 * math.pi / n
  rhs = 6.0 * (np.roll(y, -1) - 2.0 * y + np.roll(y, 1)) / h
  # circulant h (M[i-1] + 4 M[i] + M[i+1]) = rhs, eigenvalues h (4 + 2 cos w)
  w = 2.0 * math.pi * np.arange(n) / n
  m = np.real(np.fft.ifft(np.fft.fft(rhs) / (h * (4.0 + 2.0 * np.cos(w)))))
  return (np.roll(y, -1) - y) / h - h / 6.0 * (2.0 * m + np.roll(m, -1))


_HERMITE = np.array([[1.0, 0.0, 0.0, 0.0],
                     [0.0, 0.0, 1.0, 0.0],
                     [-3.0, 3.0, -2.0, -1.0],
                     [2.0, -2.0, 1.0, 1.0]])


def cmap_coefficients(grid_psi_phi) -> np.ndarray:
  """(G, G, 16) coefficients c[a*4+b] of u^a v^b (u along phi) per patch,
  from one grid stored (psi, phi) as prolix's loader stores it."""
  e = np.asarray(grid_psi_phi, dtype=np.float64).T  # (phi, psi)
  g = e.shape[0]
  d1 = np.apply_along_axis(_periodic_spline_slopes, 0, e)
  d2 = np.apply_along_axis(_periodic_spline_slopes, 1, e)
  d12 = np.apply_along_axis(_periodic_spline_slopes, 0, d2)
  delta = 2.0 * math.pi / g
  ip = (np.arange(g) + 1) % g
  out = np.empty((g, g, 16))
  for i in range(g):
    ni = ip[i]
    for j in range(g):
      nj = ip[j]
      f = np.array([
          [e[i, j], e[i, nj], d2[i, j] * delta, d2[i, nj] * delta],
          [e[ni, j], e[ni, nj], d2[ni, j] * delta, d2[ni, nj] * delta],
          [d1[i, j] * delta, d1[i, nj] * delta, d12[i, j] * delta ** 2, d12[i, nj] * delta ** 2],
          [d1[ni, j] * delta, d1[ni, nj] * delta, d12[ni, j] * delta ** 2, d12[ni, nj] * delta ** 2],
      ])
      out[i, j] = (_HERMITE @ f @ _HERMITE.T).reshape(16)
  return out
