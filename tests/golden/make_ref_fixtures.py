"""Writes ``ref_fixtures.npz``: energies, forces, Born radii and exclusion
tables computed by prolix's OWN source code, so that the FP64 oracle and
the CUDA path are both checked against the reference itself.

Run from the repository root in a container that holds the prolix sources
(default ``/root/reference/src``, or ``PROLIX_REFERENCE_SRC``):

    python tests/golden/make_ref_fixtures.py

The reference's force-field files run unmodified (``ref_loader``) on a
NumPy stand-in for JAX in FP64 (``ref_shim/``).  Which reference function
makes each value:

* exclusion table: ``ExclusionSpec.from_protein`` and
  ``map_exclusions_to_dense_padded`` (physics/neighbor_list.py:52-303);
* bond, Urey-Bradley: ``make_bond_energy_fn`` (bonded.py:20-44, jax-md's
  ``simple_spring_bond`` restated in the stand-in); angle
  ``make_angle_energy_fn`` (:47-81); torsions and periodic impropers
  ``make_dihedral_energy_fn`` (:110-141); harmonic impropers
  ``make_harmonic_improper_energy_fn`` (:144-185); exception pairs
  ``make_exception_pair_energy_fn`` (:188-230);
* CMAP: ``precompute_cmap_coefficients`` and ``compute_cmap_energy`` on
  ``compute_dihedral_angles`` of rows 0-3 / 1-4 (cmap.py:216-389,
  system.py:97-102);
* LJ, Coulomb: ``chunked_lj_energy``, ``chunked_coulomb_energy``
  (optimization.py:21-297) with the tables above; their forces from the
  reference's own hand-written backward rules (``_chunked_lj_bwd``,
  ``_chunked_coulomb_bwd``);
* GB polar and Born radii: ``compute_gb_energy`` with the dense
  ``1 - eye`` mask that make_energy_fn passes (system.py:196-207); ACE:
  ``compute_ace_nonpolar_energy`` (generalized_born.py:600-648);
* the NL-Born + dense-GB split: ``compute_born_radii_neighbor_list`` and the
  forward of ``gb_energy_split_vjp`` (generalized_born.py:266-337, :706-770)
  with the rows of every pair within the Born cutoff;
* the remaining forces (GB + ACE, and the bonded terms together) by a
  fourth-order central difference of those reference energies,
  h = 1e-4 A.  The difference is checked below against the reference's
  analytic LJ backward rule (agreement ~1e-10); where h straddles a kink
  of the reference's functions (the OBC integral's switch at
  r = rho~_i + s_j, a CMAP patch edge, the harmonic improper's wrap) the
  error grows with h, which is why h is small.

Terms are assembled as ``make_energy_fn(..., implicit_solvent=True)``
assembles them (system.py:218-244): GB all pairs, LJ and Coulomb with the
case's cutoff (0: all pairs).  The real-protein case (1A00 chain A, from
prolix's tests/physics/data/1a00.pqr) has GB, Born radii and ACE only, and
its inputs are stored with the outputs.
"""

from __future__ import annotations

import concurrent.futures
import multiprocessing
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
  sys.path.insert(0, HERE)

import ref_cases  # noqa: E402
import ref_loader  # noqa: E402

K_COULOMB = 332.0637  # physics/system.py:135
FD_H = 1e-4
PQR = "tests/physics/data/1a00.pqr"
TERMS = ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar", "exception",
         "improper", "urey_bradley")
BONDED_GROUP = ("bond", "angle", "dihedral", "improper", "urey_bradley", "cmap", "exception")
GB_GROUP = ("gb", "nonpolar")

_M = None  # reference modules, per process


def _mods():
  global _M
  if _M is None:
    _M = ref_loader.load()
  return _M


def _protein(s, explicit=None):
  """The fields ExclusionSpec.from_protein reads from a proxide Protein."""
  p = types.SimpleNamespace(charges=np.asarray(s["charges"]), bonds=np.asarray(s["bonds"]),
                            coulomb14scale=None, lj14scale=None, pairs_14=None,
                            exception_14_params=None)
  if explicit is not None:
    p.pairs_14, p.exception_14_params = explicit
  return p


class RefCase:
  """One system, evaluated term by term with the reference's functions."""

  def __init__(self, s, cutoff, explicit=None):
    m = _mods()
    from jax_md import space
    self.disp, _ = space.free()
    self.s, self.cutoff = s, float(cutoff)
    nl = m["neighbor_list"]
    self.spec = nl.ExclusionSpec.from_protein(_protein(s, explicit))
    self.excl = nl.map_exclusions_to_dense_padded(self.spec, max_exclusions=32)
    b = m["bonded"]
    d = self.disp
    self.fn = {}
    self.fn["bond"] = lambda r: b.make_bond_energy_fn(d, s["bonds"])(r, s["bond_params"])
    self.fn["angle"] = lambda r: b.make_angle_energy_fn(d, s["angles"])(r, s["angle_params"])
    self.fn["dihedral"] = lambda r: b.make_dihedral_energy_fn(d, s["dihedrals"])(r, s["dihedral_params"])
    if "impropers" in s:
      ip = np.asarray(s["improper_params"])
      maker = b.make_harmonic_improper_energy_fn if ip.shape[-1] == 2 else b.make_dihedral_energy_fn
      self.fn["improper"] = lambda r: maker(d, s["impropers"])(r, ip)
      self.fn["urey_bradley"] = lambda r: b.make_bond_energy_fn(d, s["urey_bradley_bonds"])(
          r, s["urey_bradley_params"])
    else:
      self.fn["improper"] = self.fn["urey_bradley"] = lambda r: 0.0
    if "cmap_torsions" in s:
      cm = m["cmap"]
      grids = np.asarray(s["cmap_energy_grids"], np.float64)
      self.cmap_coeffs = np.asarray(cm.precompute_cmap_coefficients(grids))
      rows = np.asarray(s["cmap_torsions"])

      def cmap_e(r, coeffs=self.cmap_coeffs):
        phi = b.compute_dihedral_angles(r, rows[:, 0:4], d)
        psi = b.compute_dihedral_angles(r, rows[:, 1:5], d)
        return cm.compute_cmap_energy(phi, psi, np.asarray(s["cmap_indices"]), coeffs)
      self.fn["cmap"] = cmap_e
      # the precomputed coefficients give make_energy_fn's per-call result
      r0 = np.asarray(s["positions"])
      direct = float(cmap_e(r0, grids))
      assert abs(direct - float(cmap_e(r0))) <= 1e-12 * max(1.0, abs(direct))
    else:
      self.cmap_coeffs = None
      self.fn["cmap"] = lambda r: 0.0
    if self.spec.exception_pairs.shape[0]:
      sp = self.spec
      ex = b.make_exception_pair_energy_fn(d, sp.exception_pairs, sp.exception_sigmas,
                                           sp.exception_epsilons, sp.exception_chargeprods)
      self.fn["exception"] = lambda r: ex(r)
    else:
      self.fn["exception"] = lambda r: 0.0

  def sig(self):
    return np.maximum(np.asarray(self.s["sigmas"], np.float64), 1e-6)  # system.py:107

  def lj(self, r):
    idx, sv, _ = self.excl
    return _mods()["optimization"].chunked_lj_energy(
        r, self.sig(), np.asarray(self.s["epsilons"], np.float64), idx, sv, self.disp, self.cutoff, 128)

  def coulomb(self, r):
    idx, _, se = self.excl
    return _mods()["optimization"].chunked_coulomb_energy(
        r, np.asarray(self.s["charges"], np.float64), idx, se, self.disp, 0.0, K_COULOMB,
        self.cutoff, 128)

  def gb(self, r):
    g = _mods()["generalized_born"]
    n = r.shape[0]
    e_gb, born = g.compute_gb_energy(r, np.asarray(self.s["charges"], np.float64),
                                     np.asarray(self.s["radii"], np.float64),
                                     mask=1.0 - np.eye(n), energy_mask=None,
                                     scaled_radii=np.asarray(self.s["scaled_radii"], np.float64))
    e_ace = np.sum(g.compute_ace_nonpolar_energy(np.asarray(self.s["radii"], np.float64), born))
    return float(e_gb), float(e_ace), np.asarray(born)

  def group_energy(self, r, group):
    if group == "gb":
      e_gb, e_ace, _ = self.gb(r)
      return e_gb + e_ace
    return float(sum(float(self.fn[t](r)) for t in BONDED_GROUP))

  def lj_forces(self, r):
    o = _mods()["optimization"]
    idx, sv, _ = self.excl
    eps = np.asarray(self.s["epsilons"], np.float64)
    res = (r, self.sig(), eps, sv)
    return -np.asarray(o.chunked_lj_energy.bwd(idx, self.disp, self.cutoff, 128, res, 1.0)[0])

  def coulomb_forces(self, r):
    o = _mods()["optimization"]
    idx, _, se = self.excl
    q = np.asarray(self.s["charges"], np.float64)
    res = (r, q, idx, se, 0.0)
    return -np.asarray(o.chunked_coulomb_energy.bwd(idx, self.disp, 0.0, K_COULOMB, self.cutoff,
                                                    128, res, 1.0)[0])


_CASE = None


def _init_worker(kind, payload):
  global _CASE
  np.seterr(divide="ignore", invalid="ignore")
  _CASE = _build_case(kind, payload)


class _JaxGather(np.ndarray):
  """An array whose integer-array indexing clamps out-of-range indices to
  the last row, as a JAX gather does (the reference's NL functions index
  positions with rows padded by N and mask those entries afterwards)."""

  def __getitem__(self, idx):
    if isinstance(idx, np.ndarray) and idx.dtype.kind in "iu":
      idx = np.clip(idx, 0, self.shape[0] - 1)
    return np.asarray(np.ndarray.__getitem__(self, idx))


class SplitCase:
  """The NL-Born + dense-GB split: ``gb_energy_split_vjp``'s forward
  (NL Born radii, then the dense GB sum) plus ACE on the same radii."""

  def __init__(self):
    s, _ = ref_cases.case_system(ref_cases.SPLIT_BASE)
    self.s = s
    r = np.asarray(s["positions"], np.float64)
    self.cutoff = ref_cases.split_cutoff(r)
    self.nbr = ref_cases.split_neighbors(r, self.cutoff)

  def terms(self, r):
    g = _mods()["generalized_born"]
    q = np.asarray(self.s["charges"], np.float64)
    rad = np.asarray(self.s["radii"], np.float64)
    sr = np.asarray(self.s["scaled_radii"], np.float64)
    rg = np.asarray(r, np.float64).view(_JaxGather)
    born = np.asarray(g.compute_born_radii_neighbor_list(rg, rad, self.nbr, scaled_radii=sr))
    e_gb = float(g.gb_energy_split_vjp(rg, q, rad, self.nbr, sr))
    e_ace = float(np.sum(g.compute_ace_nonpolar_energy(rad, born)))
    return e_gb, e_ace, born

  def group_energy(self, r, group):
    e_gb, e_ace, _ = self.terms(r)
    return e_gb + e_ace


def _build_case(kind, payload):
  if kind == "synthetic":
    s, cutoff = ref_cases.case_system(payload)
    explicit = ref_cases.exception_table(s) if ref_cases.CASES[payload][5] == "exceptions" else None
    return RefCase(s, cutoff, explicit)
  if kind == "split":
    return SplitCase()
  raise ValueError(kind)


def _fd_chunk(args):
  """-dE/dx of one energy group for the coordinates in ``coords``."""
  group, coords, r0, h = args
  out = []
  for (a, c) in coords:
    vals = []
    for k in (-2, -1, 1, 2):
      r = np.array(r0, copy=True)
      r[a, c] += k * h
      vals.append(_CASE.group_energy(r, group))
    em2, em1, ep1, ep2 = vals
    out.append(-(8.0 * (ep1 - em1) - (ep2 - em2)) / (12.0 * h))
  return out


def fd_forces(kind, payload, group, r0, workers, h=FD_H):
  n = r0.shape[0]
  coords = [(a, c) for a in range(n) for c in range(3)]
  chunks = [coords[i::workers * 4] for i in range(workers * 4)]
  ctx = multiprocessing.get_context("spawn")
  with concurrent.futures.ProcessPoolExecutor(workers, mp_context=ctx, initializer=_init_worker,
                                              initargs=(kind, payload)) as ex:
    results = list(ex.map(_fd_chunk, [(group, ch, r0, h) for ch in chunks]))
  f = np.zeros((n, 3))
  for ch, vals in zip(chunks, results):
    for (a, c), v in zip(ch, vals):
      f[a, c] = v
  return f


def synthetic_case(name, workers):
  t0 = time.time()
  case = _build_case("synthetic", name)
  s = case.s
  r = np.asarray(s["positions"], np.float64)
  e = {t: float(case.fn[t](r)) for t in BONDED_GROUP}
  e["lj"] = float(case.lj(r))
  e["coulomb"] = float(case.coulomb(r))
  e["gb"], e["nonpolar"], born = case.gb(r)
  f_lj = case.lj_forces(r)
  f_coul = case.coulomb_forces(r)
  f_gb = fd_forces("synthetic", name, "gb", r, workers)
  f_bonded = fd_forces("synthetic", name, "bonded", r, workers)
  out = {
      "terms": np.array([e[t] for t in TERMS] + [sum(e[t] for t in TERMS)]),
      "born_radii": born,
      "forces": f_lj + f_coul + f_gb + f_bonded,
      "forces_lj": f_lj, "forces_coulomb": f_coul, "forces_gb_ace": f_gb,
      "forces_bonded": f_bonded,
      "excl_indices": np.asarray(case.excl[0], np.int32),
      "excl_scales_vdw": np.asarray(case.excl[1], np.float64),
      "excl_scales_elec": np.asarray(case.excl[2], np.float64),
      "input_digest": np.array(ref_cases.digest(r, s["charges"], s["sigmas"], s["epsilons"],
                                                s["radii"], s["scaled_radii"])),
      "cutoff": np.array(case.cutoff),
  }
  if case.cmap_coeffs is not None:
    out["cmap_coeffs"] = case.cmap_coeffs
  if case.spec.exception_pairs.shape[0]:
    sp = case.spec
    out["exception_pairs"] = np.asarray(sp.exception_pairs, np.int32)
    out["exception_params"] = np.stack([np.asarray(sp.exception_chargeprods, np.float64),
                                        np.asarray(sp.exception_sigmas, np.float64),
                                        np.asarray(sp.exception_epsilons, np.float64)], axis=1)
  # self-check of the finite differences: the LJ energy's difference
  # quotient against the reference's analytic LJ backward rule, 12
  # coordinates of atoms with no pair within 5 h of a cutoff (the energy
  # jumps there, and a difference across the jump means nothing)
  rng = np.random.default_rng(0)
  worst = 0.0
  cand = np.arange(r.shape[0])
  if case.cutoff > 0:
    d = np.linalg.norm(r[:, None, :] - r[None, :, :], axis=-1)
    cand = cand[np.all(np.abs(d - case.cutoff) > 5 * FD_H, axis=1)]
  for a in rng.choice(cand, 4, replace=False):
    for c in range(3):
      vals = []
      for k in (-2, -1, 1, 2):
        rr = r.copy()
        rr[a, c] += k * FD_H
        vals.append(float(case.lj(rr)))
      fd = -(8.0 * (vals[2] - vals[1]) - (vals[3] - vals[0])) / (12.0 * FD_H)
      worst = max(worst, abs(fd - f_lj[a, c]) / max(1.0, abs(f_lj[a, c])))
  out["fd_selfcheck"] = np.array(worst)
  print(f"{name}: total {out['terms'][-1]:.8f}, FD self-check {worst:.2e}, "
        f"{time.time() - t0:.0f} s", flush=True)
  return out


def split_case(workers):
  """Born radii, GB and ACE energies of the NL-Born + dense-GB split from the
  reference's functions, and the GB + ACE forces by finite differences of
  them (the cutoff is clear of every pair distance by more than the
  difference steps, so no pair enters or leaves the list)."""
  t0 = time.time()
  case = SplitCase()
  r = np.asarray(case.s["positions"], np.float64)
  e_gb, e_ace, born = case.terms(r)
  f = fd_forces("split", None, "gb", r, workers, h=ref_cases.SPLIT_FD_H)
  print(f"{ref_cases.SPLIT_CASE}: cutoff {case.cutoff}, GB {e_gb:.8f}, ACE {e_ace:.8f}, "
        f"{time.time() - t0:.0f} s", flush=True)
  return {"born_cutoff": np.array(case.cutoff), "gb": np.array(e_gb), "nonpolar": np.array(e_ace),
          "born_radii": born, "forces_gb_ace": f,
          "input_digest": np.array(ref_cases.digest(r, case.s["charges"], case.s["radii"],
                                                    case.s["scaled_radii"]))}


def pqr_case(src):
  g = _mods()["generalized_born"]
  path = os.path.join(os.path.dirname(src.rstrip("/")), PQR)
  pos, q, rad, elem = ref_cases.read_pqr(path, "A")
  sr = ref_cases.pqr_scaled_radii(rad, elem)
  n = pos.shape[0]
  e_gb, born = g.compute_gb_energy(pos, q, rad, mask=1.0 - np.eye(n), energy_mask=None,
                                   scaled_radii=sr)
  e_ace = float(np.sum(g.compute_ace_nonpolar_energy(rad, born)))
  print(f"{ref_cases.PQR_CASE}: {n} atoms, GB {float(e_gb):.6f}, ACE {e_ace:.6f}", flush=True)
  return {"positions": pos, "charges": q, "radii": rad, "scaled_radii": sr,
          "gb": np.array(float(e_gb)), "nonpolar": np.array(e_ace), "born_radii": np.asarray(born)}


def main():
  """All cases; ``--only NAME`` recomputes one case into the existing file."""
  np.seterr(divide="ignore", invalid="ignore")  # the reference masks its own i = j divisions
  src = os.environ.get("PROLIX_REFERENCE_SRC", ref_loader.DEFAULT_SRC)
  _mods()
  workers = min(8, os.cpu_count() or 1)
  only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
  out = {"term_names": np.array(TERMS + ("total",))}
  if only is not None:
    out.update(dict(np.load(ref_cases.FIXTURE)))
  cases = [(name, lambda name=name: synthetic_case(name, workers)) for name in ref_cases.CASES]
  cases += [(ref_cases.PQR_CASE, lambda: pqr_case(src)), (ref_cases.SPLIT_CASE, lambda: split_case(workers))]
  for name, make in cases:
    if only is not None and name != only:
      continue
    for k, v in make().items():
      out[f"{name}/{k}"] = v
  np.savez_compressed(ref_cases.FIXTURE, **out)
  print(f"wrote {ref_cases.FIXTURE} ({os.path.getsize(ref_cases.FIXTURE) // 1024} KiB)")


if __name__ == "__main__":
  main()
