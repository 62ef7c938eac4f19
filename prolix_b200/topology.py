"""Host-side topology preparation: exclusion classes and CMAP patch
coefficients.

* Exclusions follow prolix's rule (utils/topology.py:26-93,
  physics/neighbor_list.py:52-142): pairs one, two or three bonds apart,
  each at its shortest separation; 1-2 and 1-3 pairs are excluded from
  Coulomb and LJ, 1-4 pairs are scaled.  Computed here with sparse
  adjacency powers: a pair joined by a walk of length k and by none shorter
  is a 1-(k+1) pair.
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
import scipy.sparse as sp

LJ14_DEFAULT = float(np.float32(0.5))
COUL14_DEFAULT = float(np.float32(0.83333333))


def exclusion_pairs(bonds, n_atoms: int):
  """(pairs (M, 2) int32 with i < j, kind (M,) int32: 0 = 1-2/1-3, 1 = 1-4)."""
  bonds = np.asarray(bonds, dtype=np.int64).reshape(-1, 2)
  if bonds.shape[0] == 0 or n_atoms < 2:
    return np.zeros((0, 2), np.int32), np.zeros(0, np.int32)
  a = sp.coo_matrix((np.ones(2 * len(bonds), dtype=np.int8),
                     (np.concatenate([bonds[:, 0], bonds[:, 1]]),
                      np.concatenate([bonds[:, 1], bonds[:, 0]]))),
                    shape=(n_atoms, n_atoms)).tocsr()
  a.data[:] = 1
  a2 = (a @ a).tocsr()
  a3 = (a2 @ a).tocsr()

  def upper_pairs(m):
    m = sp.triu(m, k=1).tocoo()
    keep = m.data != 0
    return set(zip(m.row[keep].tolist(), m.col[keep].tolist()))

  s12 = upper_pairs(a)
  s13 = upper_pairs(a2) - s12
  s14 = upper_pairs(a3) - s12 - s13
  rows = [(i, j, 0) for (i, j) in s12 | s13] + [(i, j, 1) for (i, j) in s14]
  rows.sort()
  arr = np.array(rows, dtype=np.int64).reshape(-1, 3)
  return arr[:, :2].astype(np.int32), arr[:, 2].astype(np.int32)


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
