"""Nonbonded implicit-solvent terms in FP64: OBC2 Born radii, GB polar, ACE
nonpolar, Coulomb and Lennard-Jones, with analytic forces.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Reference formulas (prolix, src/prolix/physics/):

* pair integral I_ij: generalized_born.py:211-263 (OpenMM CustomGBForce OBC2
  form, L = max(rho_i~, |r - s_j|), U = r + s_j, zero unless r + s_j > rho_i~,
  floors of 1e-4 on L, U and r);
* Born radii: dense generalized_born.py:32-94 (i = j excluded, no clamps);
  neighbour-list :266-337 (radii >= 1e-6, offset radii >= 1e-4,
  1/B >= 1e-4), which ``cutoff > 0`` follows;
* GB polar: f_GB :97-115; dense energy sums every ordered pair including
  i = j (:152-206), the neighbour-list energy adds sum q_i^2 / B_i
  explicitly (:404-413); prefactor -0.5 k (1/eps_in - 1/eps_out) (:164-165);
  distances use safe_norm, sqrt(r^2 + 1e-12) (:27-29);
* ACE nonpolar: :600-648;
* Coulomb: optimization.py:200-245 (k = 332.0637 from system.py:135, scale
  from the exclusion table, hard cutoff, pme_alpha = 0);
* LJ: optimization.py:21-70 (Lorentz-Berthelot, sigma floored at 1e-6 by
  system.py:107, scale from the exclusion table, hard cutoff);
* forces: the chain rule F = -(dE/dr|_B + sum_i dE/dB_i dB_i/dr) of
  analytical_forces.py:167-292 and generalized_born.py:773-814, written out
  analytically here (and checked against finite differences in the tests).

``cutoff <= 0`` means all pairs.  With ``cutoff > 0`` every pair term (Born
integral, GB pair, Coulomb, LJ) is restricted to r < cutoff, the behaviour of
a complete neighbour list (generalized_born.py:266-415 with the list holding
exactly the pairs inside the cutoff).
"""

from __future__ import annotations

import numpy as np

from . import topology

K_COULOMB = 332.0637
OBC_ALPHA, OBC_BETA, OBC_GAMMA = 1.0, 0.8, 4.85
DIELECTRIC_OFFSET = 0.09
ACE_COEFF_KJ_NM = 28.3919551
KJ_TO_KCAL = 0.239006
SAFE_EPS = 1e-12
ROW_CHUNK = 256


def pair_integral(r, rho_off_i, sr_j):
  """I(r; rho~_i, s_j), generalized_born.py:211-263."""
  d = np.abs(r - sr_j)
  L = np.maximum(np.maximum(rho_off_i, d), 1e-4)
  U = np.maximum(r + sr_j, 1e-4)
  rs = np.maximum(r, 1e-4)
  inv_l, inv_u = 1.0 / L, 1.0 / U
  val = (0.5 * (inv_l - inv_u) + 0.25 * np.log(L / U) / rs
         + 0.125 * (r - sr_j * sr_j / rs) * (inv_u * inv_u - inv_l * inv_l))
  return np.where(r + sr_j > rho_off_i, val, 0.0)


def pair_integral_dr(r, rho_off_i, sr_j):
  """dI/dr of :func:`pair_integral` (same branches and floors)."""
  d = np.abs(r - sr_j)
  use_d = d > rho_off_i
  Lraw = np.where(use_d, d, rho_off_i)
  L = np.maximum(Lraw, 1e-4)
  dL = np.where(use_d & (Lraw > 1e-4), np.sign(r - sr_j), 0.0)
  Uraw = r + sr_j
  U = np.maximum(Uraw, 1e-4)
  dU = np.where(Uraw > 1e-4, 1.0, 0.0)
  rs = np.maximum(r, 1e-4)
  drs = np.where(r > 1e-4, 1.0, 0.0)
  inv_l, inv_u = 1.0 / L, 1.0 / U
  t1 = 0.5 * (-dL * inv_l * inv_l + dU * inv_u * inv_u)
  lg = np.log(L / U)
  t2 = 0.25 * ((dL / L - dU / U) / rs - lg * drs / (rs * rs))
  a = r - sr_j * sr_j / rs
  da = 1.0 + sr_j * sr_j * drs / (rs * rs)
  b = inv_u * inv_u - inv_l * inv_l
  db = -2.0 * dU * inv_u ** 3 + 2.0 * dL * inv_l ** 3
  t3 = 0.125 * (da * b + a * db)
  return np.where(r + sr_j > rho_off_i, t1 + t2 + t3, 0.0)


def ace_energy(radii, born):
  """Per-atom ACE energy, generalized_born.py:600-648."""
  r_nm = (radii - DIELECTRIC_OFFSET) / 10.0 + 0.009
  b_nm = born / 10.0
  return ACE_COEFF_KJ_NM * (r_nm + 0.14) ** 2 * (r_nm / b_nm) ** 6 * KJ_TO_KCAL


def _rows(n):
  for a in range(0, n, ROW_CHUNK):
    yield a, min(n, a + ROW_CHUNK)


def _block(pos, a, b):
  dx = pos[a:b, None, :] - pos[None, :, :]
  r2 = np.einsum("ijk,ijk->ij", dx, dx)
  self_mask = np.zeros(r2.shape, dtype=bool)
  idx = np.arange(a, b)
  self_mask[idx - a, idx] = True
  return dx, r2, self_mask


def born_radii(pos, radii, scaled_radii, cutoff=0.0):
  """Born radii B, the descreening sums I and dB/dI (zero where clamped)."""
  n = pos.shape[0]
  nl = cutoff > 0
  rad = np.maximum(radii, 1e-6) if nl else radii
  rho_off = rad - DIELECTRIC_OFFSET
  if nl:
    rho_off = np.maximum(rho_off, 1e-4)
  isum = np.zeros(n)
  for a, b in _rows(n):
    _, r2, selfm = _block(pos, a, b)
    r = np.sqrt(r2 + SAFE_EPS)
    m = ~selfm
    if nl:
      m &= r < cutoff
    iv = pair_integral(r, rho_off[a:b, None], scaled_radii[None, :])
    isum[a:b] = np.where(m, iv, 0.0).sum(axis=1)
  psi = rho_off * isum
  arg = OBC_ALPHA * psi - OBC_BETA * psi ** 2 + OBC_GAMMA * psi ** 3
  th = np.tanh(arg)
  denom_r = np.maximum(rad, 1e-4) if nl else rad
  inv_b = 1.0 / rho_off - th / denom_r
  clamped = np.zeros(n, dtype=bool)
  if nl:
    clamped = inv_b < 1e-4
    inv_b = np.maximum(inv_b, 1e-4)
  born = 1.0 / inv_b
  dpsi = (OBC_ALPHA - 2.0 * OBC_BETA * psi + 3.0 * OBC_GAMMA * psi ** 2) * rho_off
  dbdi = np.where(clamped, 0.0, born * born * (1.0 - th * th) / denom_r * dpsi)
  return born, isum, dbdi


def excl_dense_rows(pairs, s_vdw, s_elec, a, b, n):
  """Scale matrices (b - a, n) for rows a..b from the sparse pair table."""
  sv = np.ones((b - a, n))
  se = np.ones((b - a, n))
  if len(pairs):
    ii = np.concatenate([pairs[:, 0], pairs[:, 1]])
    jj = np.concatenate([pairs[:, 1], pairs[:, 0]])
    vv = np.concatenate([s_vdw, s_vdw])
    ee = np.concatenate([s_elec, s_elec])
    sel = (ii >= a) & (ii < b)
    sv[ii[sel] - a, jj[sel]] = vv[sel]
    se[ii[sel] - a, jj[sel]] = ee[sel]
  return sv, se


def nonbonded(system, pos, cutoff=0.0, eps_in=1.0, eps_out=78.5, k_gb=K_COULOMB,
              k_coul=K_COULOMB, lj14=topology.LJ14_SCALE, coul14=topology.COUL14_SCALE,
              ace=True, gb_cutoff=None, born_cutoff=None):
  """Energies (dict) and forces (N, 3) of GB polar, ACE, Coulomb and LJ.

  ``cutoff`` applies to Coulomb and LJ; ``gb_cutoff`` to the GB pair terms
  and the descreening sums (None: the same as ``cutoff``; 0: all pairs, as
  prolix's make_energy_fn does for GB, system.py:196-216).  ``born_cutoff``
  > 0 applies to the descreening sums and their chain rule alone (the
  NL-Born + dense-GB split, generalized_born.py:706-817).  ``ace=False``
  drops the nonpolar term (``compute_gb_energy`` alone).
  """
  pos = np.asarray(pos, dtype=np.float64)
  n = pos.shape[0]
  q = np.asarray(system["charges"], np.float64)
  sig = np.maximum(np.asarray(system["sigmas"], np.float64), 1e-6)
  eps = np.asarray(system["epsilons"], np.float64)
  radii = np.asarray(system["radii"], np.float64)
  sr = np.asarray(system["scaled_radii"], np.float64)
  if "excl_pairs" in system:
    # an explicit table (ExclusionSpec idx_12_13 -> kind 0, idx_14 -> kind 1;
    # neighbor_list.py:33-50), e.g. with 1-4 pairs moved to exception terms
    pairs = np.asarray(system["excl_pairs"], np.int64).reshape(-1, 2)
    kind = np.asarray(system["excl_kind"], np.int64).reshape(-1)
    s_v = np.where(kind == 1, lj14, 0.0)
    s_e = np.where(kind == 1, coul14, 0.0)
  else:
    pairs, s_v, s_e = topology.pair_scales(system.get("bonds", np.zeros((0, 2))), n, lj14, coul14)
  gbc = cutoff if gb_cutoff is None else gb_cutoff
  nl = gbc > 0
  bc = born_cutoff if born_cutoff is not None and born_cutoff > 0 else gbc
  nlb = bc > 0
  born, isum, dbdi = born_radii(pos, radii, sr, bc)
  rad = np.maximum(radii, 1e-6) if nlb else radii
  rho_off = rad - DIELECTRIC_OFFSET
  if nlb:
    rho_off = np.maximum(rho_off, 1e-4)
  pref = -0.5 * k_gb * (1.0 / eps_in - 1.0 / eps_out)

  e_gb = pref * np.sum(q * q / born)
  dedb = -pref * q * q / (born * born)
  ace = ace_energy(radii, born) if ace else np.zeros(n)
  e_ace = float(np.sum(ace))
  dedb = dedb - 6.0 * ace / born
  e_coul = 0.0
  e_lj = 0.0
  force = np.zeros((n, 3))

  for a, b in _rows(n):
    dx, r2, selfm = _block(pos, a, b)
    m = ~selfm
    rg = np.sqrt(r2 + SAFE_EPS)
    if nl:
      m &= rg < gbc
    # GB pair terms (every pair, no exclusions)
    bi = born[a:b, None]
    bj = born[None, :]
    dprod = bi * bj
    ex = np.exp(-rg * rg / (4.0 * dprod))
    f2 = rg * rg + dprod * ex
    f = np.sqrt(f2)
    qq = q[a:b, None] * q[None, :]
    e_gb += pref * np.sum(np.where(m, qq / f, 0.0))
    inv_f3 = 1.0 / (f2 * f)
    # d(1/f)/d r_i along (r_i - r_j)/rg, with d f/d rg = rg (1 - ex/4) / f
    g = np.where(m, 2.0 * pref * qq * (1.0 - 0.25 * ex) * inv_f3, 0.0)
    force[a:b] += np.einsum("ij,ijk->ik", g, dx)
    dedb[a:b] += np.sum(np.where(m, -pref * qq * ex * (1.0 + rg * rg / (4.0 * dprod)) * bj
                                 * inv_f3, 0.0), axis=1)
    # Coulomb / LJ with exclusion scales
    r = np.sqrt(r2)
    mc = ~selfm & (r > 0)
    if cutoff > 0:
      mc &= r < cutoff
    sv, se = excl_dense_rows(pairs, s_v, s_e, a, b, n)
    rs = np.where(mc, r, 1.0)
    inv_r = 1.0 / rs
    ec = np.where(mc, k_coul * qq * se * inv_r, 0.0)
    e_coul += 0.5 * np.sum(ec)
    gc = np.where(mc, ec * inv_r * inv_r, 0.0)
    sij = 0.5 * (sig[a:b, None] + sig[None, :])
    eij = np.sqrt(eps[a:b, None] * eps[None, :])
    s6 = (sij * inv_r) ** 6
    el = np.where(mc, 4.0 * eij * (s6 * s6 - s6) * sv, 0.0)
    e_lj += 0.5 * np.sum(el)
    gl = np.where(mc, 4.0 * eij * (12.0 * s6 * s6 - 6.0 * s6) * sv * inv_r * inv_r, 0.0)
    force[a:b] += np.einsum("ij,ijk->ik", gc + gl, dx)

  dedi = dedb * dbdi
  for a, b in _rows(n):
    dx, r2, selfm = _block(pos, a, b)
    m = ~selfm
    rg = np.sqrt(r2 + SAFE_EPS)
    if nlb:
      m &= rg < bc
    d_ij = pair_integral_dr(rg, rho_off[a:b, None], sr[None, :])
    d_ji = pair_integral_dr(rg, rho_off[None, :], sr[a:b, None])
    g = np.where(m, (dedi[a:b, None] * d_ij + dedi[None, :] * d_ji) / rg, 0.0)
    force[a:b] -= np.einsum("ij,ijk->ik", g, dx)

  energies = {"gb": float(e_gb), "nonpolar": e_ace, "coulomb": float(e_coul),
              "lj": float(e_lj)}
  extras = {"born_radii": born, "born_sum": isum, "dbdi": dbdi, "dedb": dedb}
  return energies, force, extras


def nonbonded_energy(system, pos, cutoff=0.0, **kw):
  """Energy only (for finite-difference checks)."""
  return sum(nonbonded(system, pos, cutoff, **kw)[0].values())
