"""Bonded terms and CMAP in FP64 with analytic forces.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Reference formulas (prolix, src/prolix/physics/):

* bond: jax_md ``simple_spring_bond`` as bound in bonded.py:20-44,
  E = 1/2 k (r - r0)^2 with params rows (r0, k) (typing.py:77-78);
* angle: bonded.py:47-81, cos(theta) = v_ji . v_jk / (|v_ji||v_jk| + 1e-8)
  clipped to +-0.999999, E = 1/2 k (theta - theta0)^2, rows (theta0, k);
* dihedral angle: bonded.py:84-107 (b0 = r_i - r_j, b1 = r_k - r_j,
  b2 = r_l - r_k, phi = atan2(y, x));
* periodic torsion: bonded.py:110-141, E = sum_terms k (1 + cos(n phi - delta)),
  params (D, T, 3) = (n, delta, k);
* impropers: system.py:63-88 picks the form by the parameters' last axis:
  3 -> periodic, the torsion formula above (make_dihedral_energy_fn);
  2 -> harmonic (make_harmonic_improper_energy_fn, bonded.py:144-185),
  params (M, T, 2) = (k, phi0), E = sum k d^2 with
  d = ((phi - phi0 + pi) mod 2 pi) - pi (no factor 1/2);
* Urey-Bradley: harmonic bonds between the 1-3 atoms, the bond formula
  above on (r0, k) rows (system.py:93-95);
* CMAP: cmap.py:62-389.  Grids are stored (psi, phi) and transposed to
  (phi, psi) (cmap.py:256-259); derivatives at the grid points come from
  periodic cubic splines (create_periodic_spline :62-124,
  evaluate_spline_derivative :127-163, compute_map_derivatives :166-216);
  each 2-pi/24 patch is a bicubic matching the corner values and scaled
  derivatives (compute_bicubic_coefficients :242-286); evaluation at
  angles mapped to [0, 2 pi) (compute_cmap_energies :316-376).  phi uses
  row atoms 0-3 and psi atoms 1-4 (system.py:99-102).

The bicubic coefficients here are obtained by solving the 16 corner
conditions directly rather than from a precomputed weight table: the
interpolant is the same unique bicubic.
"""

from __future__ import annotations

import math

import numpy as np


def _scatter(force, idx, contrib):
  for k in range(idx.shape[1]):
    np.add.at(force, idx[:, k], contrib[k])


def bonds(pos, idx, params):
  idx = np.asarray(idx, np.int64).reshape(-1, 2)
  params = np.asarray(params, np.float64).reshape(-1, 2)
  f = np.zeros_like(pos)
  if idx.shape[0] == 0:
    return 0.0, f
  d = pos[idx[:, 0]] - pos[idx[:, 1]]
  r = np.sqrt((d * d).sum(1))
  r0, k = params[:, 0], params[:, 1]
  e = 0.5 * k * (r - r0) ** 2
  g = (k * (r - r0) / r)[:, None] * d  # dE/dr_i
  _scatter(f, idx, [-g, g])
  return float(e.sum()), f


def angles(pos, idx, params):
  idx = np.asarray(idx, np.int64).reshape(-1, 3)
  params = np.asarray(params, np.float64).reshape(-1, 2)
  f = np.zeros_like(pos)
  if idx.shape[0] == 0:
    return 0.0, f
  ri, rj, rk = pos[idx[:, 0]], pos[idx[:, 1]], pos[idx[:, 2]]
  a = ri - rj
  b = rk - rj
  la = np.sqrt((a * a).sum(1))
  lb = np.sqrt((b * b).sum(1))
  den = la * lb + 1e-8
  dot = (a * b).sum(1)
  c = dot / den
  clipped = (c < -0.999999) | (c > 0.999999)
  c = np.clip(c, -0.999999, 0.999999)
  th = np.arccos(c)
  th0, k = params[:, 0], params[:, 1]
  e = 0.5 * k * (th - th0) ** 2
  dedth = k * (th - th0)
  dthdc = np.where(clipped, 0.0, -1.0 / np.sqrt(1.0 - c * c))
  # dc/da = b/den - dot * lb * (a/la) / den^2
  dcda = b / den[:, None] - (dot * lb / (den * den * la))[:, None] * a
  dcdb = a / den[:, None] - (dot * la / (den * den * lb))[:, None] * b
  s = (dedth * dthdc)[:, None]
  gi = s * dcda
  gk = s * dcdb
  _scatter(f, idx, [-gi, gi + gk, -gk])
  return float(e.sum()), f


def dihedral(pos, idx):
  """phi (M,) and dphi/dr for the four atoms (4, M, 3)."""
  idx = np.asarray(idx, np.int64).reshape(-1, 4)
  ri, rj, rk, rl = (pos[idx[:, c]] for c in range(4))
  b0 = ri - rj
  b1 = rk - rj
  b2 = rl - rk
  nb1 = np.sqrt((b1 * b1).sum(1, keepdims=True)) + 1e-8
  u = b1 / nb1
  v = b0 - (b0 * u).sum(1, keepdims=True) * u
  w = b2 - (b2 * u).sum(1, keepdims=True) * u
  x = (v * w).sum(1)
  y = (np.cross(u, v) * w).sum(1)
  phi = np.arctan2(y, x)
  # gradient with the standard torsion formula in terms of
  # F = r_i - r_j, G = r_j - r_k, H = r_l - r_k, A = F x G, B = H x G
  F = ri - rj
  G = rj - rk
  H = rl - rk
  A = np.cross(F, G)
  B = np.cross(H, G)
  lg = np.sqrt((G * G).sum(1))
  a2 = (A * A).sum(1)
  b2n = (B * B).sum(1)
  fg = (F * G).sum(1)
  hg = (H * G).sum(1)
  gi = -(lg / a2)[:, None] * A
  gl = (lg / b2n)[:, None] * B
  gj = -gi + (fg / (a2 * lg))[:, None] * A - (hg / (b2n * lg))[:, None] * B
  gk = -gl - (fg / (a2 * lg))[:, None] * A + (hg / (b2n * lg))[:, None] * B
  return phi, np.stack([gi, gj, gk, gl])


def torsions(pos, idx, params):
  idx = np.asarray(idx, np.int64).reshape(-1, 4)
  f = np.zeros_like(pos)
  if idx.shape[0] == 0:
    return 0.0, f
  params = np.asarray(params, np.float64).reshape(idx.shape[0], -1, 3)
  phi, dphi = dihedral(pos, idx)
  n, dl, k = params[..., 0], params[..., 1], params[..., 2]
  ang = n * phi[:, None] - dl
  e = (k * (1.0 + np.cos(ang))).sum()
  dedphi = (-k * n * np.sin(ang)).sum(1)
  _scatter(f, idx, [-(dedphi[:, None] * dphi[c]) for c in range(4)])
  return float(e), f


def harmonic_impropers(pos, idx, params):
  """k d^2, d = ((phi - phi0 + pi) mod 2 pi) - pi, params (M, T, 2) = (k, phi0)
  (bonded.py:178-183)."""
  idx = np.asarray(idx, np.int64).reshape(-1, 4)
  f = np.zeros_like(pos)
  if idx.shape[0] == 0:
    return 0.0, f
  params = np.asarray(params, np.float64).reshape(idx.shape[0], -1, 2)
  phi, dphi = dihedral(pos, idx)
  k, phi0 = params[..., 0], params[..., 1]
  d = np.mod(phi[:, None] - phi0 + np.pi, 2.0 * np.pi) - np.pi
  e = (k * d * d).sum()
  dedphi = (2.0 * k * d).sum(1)
  _scatter(f, idx, [-(dedphi[:, None] * dphi[c]) for c in range(4)])
  return float(e), f


def impropers(pos, idx, params):
  """Either improper form, chosen as system.py:77-83 does by the last axis
  of the parameters (2: harmonic, else periodic)."""
  params = np.asarray(params, np.float64)
  if params.size and params.shape[-1] == 2:
    return harmonic_impropers(pos, idx, params)
  return torsions(pos, idx, params)


def _first(system, *keys, default):
  for k in keys:
    v = system.get(k)
    if v is not None and np.asarray(v).size:
      return v
  return default


# ---------------------------------------------------------------- CMAP

def _periodic_spline_second_derivs(y):
  """Second derivatives of the periodic cubic spline through y[0..n-1] on a
  uniform grid of spacing h = 2 pi / n (cmap.py:62-124)."""
  n = y.shape[0]
  h = 2.0 * math.pi / n
  a = np.zeros((n, n))
  for i in range(n):
    a[i, i] = 4.0 * h
    a[i, (i - 1) % n] += h
    a[i, (i + 1) % n] += h
  rhs = 6.0 * (np.roll(y, -1) - 2.0 * y + np.roll(y, 1)) / h
  return np.linalg.solve(a, rhs)


def _spline_knot_derivs(y):
  """f'(x_i) of the periodic spline at each knot (cmap.py:127-163 at a=1, b=0)."""
  n = y.shape[0]
  h = 2.0 * math.pi / n
  m = _periodic_spline_second_derivs(y)
  return (np.roll(y, -1) - y) / h - h / 6.0 * (2.0 * m + np.roll(m, -1))


def _bicubic_solver():
  """Inverse of the 16 x 16 corner-condition matrix of a bicubic patch.

  Unknowns c[a*4+b] of p(u, v) = sum c_ab u^a v^b on [0,1]^2; conditions in
  the order (value, d/du, d/dv, d2/dudv) x corners (0,0), (1,0), (1,1), (0,1).
  """
  corners = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]
  rows = []
  for kind in range(4):
    for (u, v) in corners:
      row = np.zeros(16)
      for a in range(4):
        for b in range(4):
          if kind == 0:
            val = u ** a * v ** b
          elif kind == 1:
            val = a * u ** (a - 1) * v ** b if a > 0 else 0.0
          elif kind == 2:
            val = b * u ** a * v ** (b - 1) if b > 0 else 0.0
          else:
            val = a * b * u ** (a - 1) * v ** (b - 1) if (a > 0 and b > 0) else 0.0
          row[4 * a + b] = val
      rows.append(row)
  return np.linalg.inv(np.array(rows))


def cmap_coefficients(grid_psi_phi):
  """(G, G, 16) patch coefficients from one grid stored (psi, phi)."""
  e = np.asarray(grid_psi_phi, np.float64).T  # -> (phi, psi)
  g = e.shape[0]
  d1 = np.stack([_spline_knot_derivs(e[:, j]) for j in range(g)], axis=1)
  d2 = np.stack([_spline_knot_derivs(e[i, :]) for i in range(g)], axis=0)
  d12 = np.stack([_spline_knot_derivs(d2[:, j]) for j in range(g)], axis=1)
  delta = 2.0 * math.pi / g
  inv = _bicubic_solver()
  out = np.zeros((g, g, 16))
  for i in range(g):
    ni = (i + 1) % g
    for j in range(g):
      nj = (j + 1) % g
      cidx = [(i, j), (ni, j), (ni, nj), (i, nj)]
      rhs = np.array([e[c] for c in cidx] + [d1[c] * delta for c in cidx]
                     + [d2[c] * delta for c in cidx] + [d12[c] * delta * delta for c in cidx])
      out[i, j] = inv @ rhs
  return out


def cmap(pos, torsion_rows, map_idx, grids):
  rows = np.asarray(torsion_rows, np.int64).reshape(-1, 5)
  f = np.zeros_like(pos)
  if rows.shape[0] == 0:
    return 0.0, f
  grids = np.asarray(grids, np.float64)
  coeffs = np.stack([cmap_coefficients(gr) for gr in grids])
  g = grids.shape[1]
  delta = 2.0 * math.pi / g
  phi, dphi = dihedral(pos, rows[:, 0:4])
  psi, dpsi = dihedral(pos, rows[:, 1:5])
  pn = np.mod(phi + 2.0 * math.pi, 2.0 * math.pi)
  sn = np.mod(psi + 2.0 * math.pi, 2.0 * math.pi)
  i = np.floor(pn / delta).astype(np.int64) % g
  j = np.floor(sn / delta).astype(np.int64) % g
  da = pn / delta - i
  db = sn / delta - j
  c = coeffs[np.asarray(map_idx, np.int64), i, j].reshape(-1, 4, 4)
  pa = np.stack([np.ones_like(da), da, da ** 2, da ** 3], 1)
  pb = np.stack([np.ones_like(db), db, db ** 2, db ** 3], 1)
  dpa = np.stack([np.zeros_like(da), np.ones_like(da), 2 * da, 3 * da ** 2], 1)
  dpb = np.stack([np.zeros_like(db), np.ones_like(db), 2 * db, 3 * db ** 2], 1)
  e = np.einsum("ta,tab,tb->t", pa, c, pb)
  dedphi = np.einsum("ta,tab,tb->t", dpa, c, pb) / delta
  dedpsi = np.einsum("ta,tab,tb->t", pa, c, dpb) / delta
  for k in range(4):
    np.add.at(f, rows[:, k], -dedphi[:, None] * dphi[k])
    np.add.at(f, rows[:, k + 1], -dedpsi[:, None] * dpsi[k])
  return float(e.sum()), f


def exception_pairs(pos, pairs, sigmas, epsilons, chargeprods, k_coul=332.0637):
  """Explicit 1-4 exception pairs (prolix bonded.py:186-230): per pair, with
  parameters already scaled, d = sqrt(|r_i - r_j|^2 + 1e-12) and
  E = 4 eps ((sigma/d)^12 - (sigma/d)^6) + k_coul qq / d.  Returns
  (energy, forces)."""
  pos = np.asarray(pos, np.float64)
  f = np.zeros_like(pos)
  pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
  if pairs.shape[0] == 0:
    return 0.0, f
  sig = np.asarray(sigmas, np.float64)
  eps = np.asarray(epsilons, np.float64)
  qq = np.asarray(chargeprods, np.float64)
  dr = pos[pairs[:, 0]] - pos[pairs[:, 1]]
  d = np.sqrt(np.sum(dr * dr, axis=1) + 1e-12)
  s6 = (sig / d) ** 6
  e_lj = 4.0 * eps * (s6 * s6 - s6)
  e_c = k_coul * qq / d
  dedd = (4.0 * eps * (-12.0 * s6 * s6 + 6.0 * s6) - e_c) / d
  g = (dedd / d)[:, None] * dr  # dE/dr_i
  np.add.at(f, pairs[:, 0], -g)
  np.add.at(f, pairs[:, 1], g)
  return float(np.sum(e_lj + e_c)), f


def bonded_all(system, pos):
  """Energies (dict: bond, angle, dihedral, improper, urey_bradley, cmap)
  and the summed force.  Key names as make_energy_fn reads them
  (system.py:46-95): ``dihedrals`` or ``proper_dihedrals``, ``impropers``
  or ``improper_dihedrals`` with ``improper_params`` or
  ``improper_dihedral_params``, ``urey_bradley_bonds`` /
  ``urey_bradley_params``."""
  pos = np.asarray(pos, np.float64)
  eb, fb = bonds(pos, system.get("bonds", np.zeros((0, 2))),
                 system.get("bond_params", np.zeros((0, 2))))
  ea, fa = angles(pos, system.get("angles", np.zeros((0, 3))),
                  system.get("angle_params", np.zeros((0, 2))))
  ed, fd = torsions(pos, _first(system, "dihedrals", "proper_dihedrals", default=np.zeros((0, 4))),
                    _first(system, "dihedral_params", "proper_dihedral_params",
                           default=np.zeros((0, 1, 3))))
  ei, fi = impropers(pos, _first(system, "impropers", "improper_dihedrals", default=np.zeros((0, 4))),
                     _first(system, "improper_params", "improper_dihedral_params",
                            default=np.zeros((0, 1, 3))))
  eu, fu = bonds(pos, _first(system, "urey_bradley_bonds", default=np.zeros((0, 2))),
                 _first(system, "urey_bradley_params", default=np.zeros((0, 2))))
  if "cmap_torsions" in system:
    ec, fc = cmap(pos, system["cmap_torsions"], system["cmap_indices"],
                  system["cmap_energy_grids"])
  else:
    ec, fc = 0.0, np.zeros_like(pos)
  return ({"bond": eb, "angle": ea, "dihedral": ed, "improper": ei, "urey_bradley": eu, "cmap": ec},
          fb + fa + fd + fi + fu + fc)
