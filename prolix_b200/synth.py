"""Seeded synthetic peptide-like chains (the benchmark and test inputs).

Every system is drawn from ``numpy.random.default_rng(seed)`` in a fixed
order, so a seed names one system exactly:

* geometry: a self-avoiding chain with bond lengths U(1.0, 1.53) A, bond
  angles U(105, 120) deg and random dihedrals; atoms three or more bonds apart
  stay at least 2.5 A apart where the packing allows.  ``compact=True`` keeps
  the chain inside a sphere of radius (3N / (4 pi 0.075))^(1/3) A where it
  can (20 A at N=2,500; 40 A at N=20,000), giving a compact globule;
* charges U(-0.8, 0.8) e shifted to net zero; LJ sigma U(1.0, 3.4) A and
  epsilon U(0.01, 0.2) kcal/mol (ranges adjustable: with these, two
  opposite charges on small-sigma sites can meet in a ~0.5 A well, so
  constant-energy runs start from a minimised, thermalised state); GB
  intrinsic radii U(1.2, 1.9) A and OBC
  scale factors U(0.72, 0.85), with ``scaled_radii = radii * scale``
  (the convention of prolix tests/physics/test_openmm_parity.py:113);
* masses drawn from {1.008, 12.011, 14.007, 15.999} amu;
* topology: bonds (i, i+1) with k U(300, 500) and r0 the generated length,
  angles (i, i+1, i+2) with k U(50, 100) and theta0 the generated angle,
  one periodic torsion term per (i..i+3) with n in {1, 2, 3}, phase in
  {0, pi} and k U(0.1, 2.0);
* optional CMAP: one 5-atom (phi, psi) row per 16-atom residue and one
  24 x 24 grid of U(-2, 2) kcal/mol values, stored (psi, phi) as prolix's
  force-field loader stores them (prolix physics/cmap.py:256-259).

The returned dict uses the keys that prolix's ``PhysicsSystem.from_dict``
reads (prolix typing.py:357-425) plus ``positions`` and CMAP fields.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _host

MASS_CHOICES = np.array([1.008, 12.011, 14.007, 15.999])
GLOBULE_DENSITY = 0.075  # atoms / A^3
N_CANDIDATES = 32
MIN_NONBONDED_DIST = 2.5


def globule_radius(n_atoms: int, density: float = GLOBULE_DENSITY) -> float:
  """Radius of a sphere holding ``n_atoms`` at ``density``."""
  return (3.0 * n_atoms / (4.0 * math.pi * density)) ** (1.0 / 3.0)


def _grow(lengths, angles, cand, compact, confine, retry_seed):
  lib = _host.lib()
  n = lengths.shape[0]
  pos = np.zeros((n, 3), dtype=np.float64)
  chosen = np.zeros(n, dtype=np.float64)
  dp = ctypes.POINTER(ctypes.c_double)
  rc = lib.pb2_synth_grow_chain(
      ctypes.c_int(n), ctypes.c_int(cand.shape[1]),
      lengths.ctypes.data_as(dp), angles.ctypes.data_as(dp), cand.ctypes.data_as(dp),
      ctypes.c_int(1 if compact else 0), ctypes.c_double(confine),
      ctypes.c_double(MIN_NONBONDED_DIST), ctypes.c_ulonglong(retry_seed),
      pos.ctypes.data_as(dp), chosen.ctypes.data_as(dp))
  if rc < 0:
    raise MemoryError("chain growth could not allocate its grid")
  return pos, chosen, rc


# Parameter ranges with a real LJ core on every site.  With the default
# ranges (|q| <= 0.8 e, sigma from 1 A) opposite charges meet in ~0.55 A
# wells whose compressed LJ wall has omega * dt > 2 for hydrogen masses even
# at 0.5 fs: nearly every system of a 512-system batch passes 1,000 K within
# 100 Langevin steps at 1 fs.  Dynamics workloads (timing, serving, energy
# drift) use these ranges instead; the draw order is unchanged.
PHYSICAL_RANGES = {"charge_range": (-0.5, 0.5), "sigma_range": (2.4, 3.4), "eps_range": (0.03, 0.2)}


def make_chain(n_atoms: int, seed: int, *, compact: bool = False, cmap: bool = False,
               n_cmap_maps: int = 1, cmap_grid: int = 24, charge_range=(-0.8, 0.8),
               sigma_range=(1.0, 3.4), eps_range=(0.01, 0.2)) -> dict:
  """Build one seeded synthetic system of ``n_atoms`` atoms."""
  if n_atoms < 1:
    raise ValueError("n_atoms must be >= 1")
  rng = np.random.default_rng(seed)
  n = int(n_atoms)
  lengths = rng.uniform(1.0, 1.53, size=n)
  angles = np.deg2rad(rng.uniform(105.0, 120.0, size=n))
  cand = rng.uniform(-math.pi, math.pi, size=(n, N_CANDIDATES))
  retry_seed = int(rng.integers(0, 2**63))
  pos, _, _ = _grow(lengths, angles, cand, compact, globule_radius(n), retry_seed)
  pos = pos - pos.mean(axis=0, keepdims=True)

  q = rng.uniform(*charge_range, size=n)
  q = q - q.mean()
  sigma = rng.uniform(*sigma_range, size=n)
  eps = rng.uniform(*eps_range, size=n)
  radii = rng.uniform(1.2, 1.9, size=n)
  scale = rng.uniform(0.72, 0.85, size=n)
  masses = MASS_CHOICES[rng.integers(0, 4, size=n)]

  nb = max(n - 1, 0)
  bonds = np.stack([np.arange(nb), np.arange(1, nb + 1)], axis=1).astype(np.int32)
  bond_k = rng.uniform(300.0, 500.0, size=nb)
  bond_params = np.stack([lengths[1:n], bond_k], axis=1) if nb else np.zeros((0, 2))

  na = max(n - 2, 0)
  angle_idx = np.stack([np.arange(na), np.arange(1, na + 1), np.arange(2, na + 2)],
                       axis=1).astype(np.int32)
  angle_k = rng.uniform(50.0, 100.0, size=na)
  angle_params = np.stack([angles[2:n], angle_k], axis=1) if na else np.zeros((0, 2))

  nd = max(n - 3, 0)
  dih_idx = np.stack([np.arange(nd) + o for o in range(4)], axis=1).astype(np.int32)
  per = rng.integers(1, 4, size=nd).astype(np.float64)
  phase = np.where(rng.integers(0, 2, size=nd) == 1, math.pi, 0.0)
  tk = rng.uniform(0.1, 2.0, size=nd)
  dih_params = np.stack([per, phase, tk], axis=1)[:, None, :] if nd else np.zeros((0, 1, 3))

  system = {
      "positions": pos,
      "charges": q,
      "sigmas": sigma,
      "epsilons": eps,
      "radii": radii,
      "scaled_radii": radii * scale,
      "masses": masses,
      "bonds": bonds,
      "bond_params": bond_params,
      "angles": angle_idx,
      "angle_params": angle_params,
      "dihedrals": dih_idx,
      "dihedral_params": dih_params,
      "seed": int(seed),
  }
  if cmap:
    n_res = n // 16
    rows = [np.arange(16 * r + 1, 16 * r + 6) for r in range(n_res) if 16 * r + 5 < n]
    tors = np.array(rows, dtype=np.int32).reshape(-1, 5)
    grids = rng.uniform(-2.0, 2.0, size=(n_cmap_maps, cmap_grid, cmap_grid))
    idx = rng.integers(0, n_cmap_maps, size=tors.shape[0]).astype(np.int32)
    system["cmap_torsions"] = tors
    system["cmap_indices"] = idx
    system["cmap_energy_grids"] = grids
  return system


def batch_sizes(n_systems: int, seed: int, lo: int = 150, hi: int = 4000) -> np.ndarray:
  """Atom counts log-uniform in [lo, hi], seeded (the ragged-batch workload)."""
  rng = np.random.default_rng(seed)
  return np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_systems)).astype(np.int64)


def make_batch(n_systems: int, seed: int, lo: int = 150, hi: int = 4000, *,
               compact: bool = True, cmap: bool = False, **ranges) -> list[dict]:
  """``n_systems`` systems with log-uniform sizes; system k uses seed
  ``seed + 1 + k``; ``ranges`` as make_chain's (e.g. PHYSICAL_RANGES)."""
  sizes = batch_sizes(n_systems, seed, lo, hi)
  return [make_chain(int(n), seed + 1 + k, compact=compact, cmap=cmap, **ranges)
          for k, n in enumerate(sizes)]
