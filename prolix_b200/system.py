"""Drop-in for prolix's energy factory on the implicit-solvent path.

``make_energy_fn(displacement_fn, system, cutoff_distance=9.0,
return_decomposed=False, implicit_solvent=False, exclusion_spec=None, **kw)``
mirrors prolix physics/system.py:29-271 for ``implicit_solvent=True``:

* GB polar (with self term) and the OBC2 Born radii use every pair, and
  Coulomb and LJ use ``cutoff`` (the ``cutoff`` keyword wins over
  ``cutoff_distance``, system.py:134; a cutoff <= 0 means all pairs), as the
  reference does (system.py:184-216);
* exclusions come from ``exclusion_spec`` (an ExclusionSpec or any object
  with its fields; ``exclusion_spec_from_bonds`` builds one from a bond
  list as ``ExclusionSpec.from_protein`` does) or from the system's own
  ``excl_indices`` / ``excl_scales_vdw`` / ``excl_scales_elec`` table
  (system.py:161-171).  With neither, Coulomb and LJ exclude no pair at
  all: the reference then uses an empty (N, 0) table;
* bonded terms: bonds, angles, dihedrals (or ``proper_dihedrals``),
  impropers (``impropers`` or ``improper_dihedrals``; parameter rows of 2
  values are harmonic (k, phi0), of 3 periodic (n, phase, k), as
  system.py:77-83 decides), Urey-Bradley springs, CMAP and the
  exclusion spec's explicit 1-4 exception pairs;
* a dict key this path does not read raises ``ValueError`` (rather than
  being dropped), except metadata the reference's energy factory ignores
  too (masks of bonded terms, element and selection flags, constraint
  and water tables);
* the returned function gives the total energy; ``.forces(r)`` gives
  -dE/dr, ``.energy_and_forces(r)`` both;
* ``return_decomposed=True`` returns the reference's dict of per-term
  callables (system.py:250-270).

Positions are NumPy arrays (N, 3) in A; free space only (prolix's implicit
runs use ``space.free()``).  Everything runs on the GPU through the C ABI.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from . import engine, topology
from ._lib import TERM_NAMES, USE_ALL

_SYSTEM_KEYS = ("charges", "sigmas", "epsilons", "radii", "scaled_radii", "masses", "bonds",
                "bond_params", "angles", "angle_params", "dihedrals", "dihedral_params",
                "proper_dihedrals", "proper_dihedral_params", "impropers", "improper_params",
                "improper_dihedrals", "improper_dihedral_params", "urey_bradley_bonds",
                "urey_bradley_params", "cmap_torsions", "cmap_indices",
                "cmap_energy_grids", "excl_indices", "excl_scales_vdw", "excl_scales_elec",
                "excl_pairs", "excl_kind", "exception_pairs",
                "exception_sigmas", "exception_epsilons", "exception_chargeprods", "atom_mask")
# keys read by the batch itself (integrator settings, explicit 1-4 scales, origin)
_ENGINE_KEYS = ("positions", "lj14_scale", "coul14_scale", "key", "seed", "dt", "kT", "gamma",
                "origin", "solute_dielectric", "solvent_dielectric")
# PhysicsSystem fields the reference's energy factory does not read either
# (typing.py:256-336 against system.py:29-271): masks of bonded terms, atom
# flags, constraint / water tables, the dense exclusion matrix, padding
# metadata
_IGNORED_KEYS = ("element_ids", "is_hydrogen", "is_backbone", "is_heavy", "protein_atom_mask",
                 "water_atom_mask", "bond_mask", "angle_mask", "dihedral_mask", "improper_mask",
                 "urey_bradley_mask", "cmap_mask", "constraint_pairs", "constraint_lengths",
                 "constraint_mask", "water_indices", "water_mask", "n_real_atoms",
                 "n_padded_atoms", "bucket_size", "box_size", "exclusion_mask",
                 "nonbonded_cutoff", "pme_alpha", "pme_grid_points", "atom_names",
                 "residue_names", "residue_index", "cmap_coeffs")


def system_to_dict(system) -> dict:
  """Accept a dict or any object with prolix's PhysicsSystem attribute names.

  A dict key that is neither read here nor ignored by the reference's
  energy factory raises ``ValueError``; so does an ``atom_mask`` with
  padding atoms (the reference zeroes their ACE term, system.py:230; a
  batch holds real atoms only)."""
  if isinstance(system, dict):
    unknown = sorted(set(system) - set(_SYSTEM_KEYS) - set(_ENGINE_KEYS) - set(_IGNORED_KEYS))
    if unknown:
      raise ValueError(f"system keys not understood by the implicit-solvent energy: {unknown}")
    out = {k: v for k, v in system.items() if k not in _IGNORED_KEYS}
  else:
    out = {}
    for k in _SYSTEM_KEYS + ("positions",):
      v = getattr(system, k, None)
      if v is not None:
        out[k] = np.asarray(v)
  mask = out.pop("atom_mask", None)
  if mask is not None and not np.all(np.asarray(mask, dtype=bool)):
    raise ValueError("atom_mask marks padding atoms; pass the real atoms only "
                     "(a batch stores systems unpadded)")
  return out


@dataclasses.dataclass(frozen=True)
class ExclusionSpec:
  """prolix's ExclusionSpec fields (physics/neighbor_list.py:25-50)."""
  idx_12_13: np.ndarray
  idx_14: np.ndarray
  scale_14_elec: float
  scale_14_vdw: float
  n_atoms: int
  exception_pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 2), np.int32))
  exception_sigmas: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
  exception_epsilons: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
  exception_chargeprods: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))


def exclusion_spec_from_bonds(bonds, n_atoms: int, coulomb14scale: float = 0.83333333,
                              lj14scale: float = 0.5) -> ExclusionSpec:
  """``ExclusionSpec.from_protein`` for a bond list without explicit 1-4
  parameters (neighbor_list.py:52-142): 1-2 and 1-3 pairs excluded, 1-4
  pairs scaled."""
  pairs, kind = topology.exclusion_pairs(bonds, n_atoms)
  return ExclusionSpec(idx_12_13=pairs[kind == 0], idx_14=pairs[kind == 1],
                       scale_14_elec=coulomb14scale, scale_14_vdw=lj14scale, n_atoms=int(n_atoms))


def _exclusions_from_spec(spec, n):
  """(pairs, kind, lj14, coul14) from a prolix ExclusionSpec-like object."""
  p1213 = np.asarray(getattr(spec, "idx_12_13", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
  p14 = np.asarray(getattr(spec, "idx_14", np.zeros((0, 2))), dtype=np.int64).reshape(-1, 2)
  rows = {}
  for (i, j) in p1213:
    a, b = (int(i), int(j)) if i < j else (int(j), int(i))
    rows[(a, b)] = 0
  for (i, j) in p14:
    a, b = (int(i), int(j)) if i < j else (int(j), int(i))
    rows.setdefault((a, b), 1)
  keys = sorted(rows)
  pairs = np.array(keys, dtype=np.int32).reshape(-1, 2)
  kind = np.array([rows[k] for k in keys], dtype=np.int32)
  lj14 = float(np.float32(getattr(spec, "scale_14_vdw", topology.LJ14_DEFAULT)))
  c14 = float(np.float32(getattr(spec, "scale_14_elec", topology.COUL14_DEFAULT)))
  return pairs, kind, lj14, c14


class EnergyFn:
  """Callable energy function backed by a one-system device batch."""

  def __init__(self, system: dict, cutoff: float, *, eps_in=1.0, eps_out=78.5,
               terms=USE_ALL, device=0, gb_cutoff=0.0, born_cutoff=0.0, **defaults):
    self.system = system
    self.cutoff = float(cutoff)
    self.gb_cutoff = float(gb_cutoff)
    self.born_cutoff = float(born_cutoff)
    self._batch = engine.Batch([system], cutoff=self.cutoff, gb_cutoff=self.gb_cutoff,
                               born_cutoff=self.born_cutoff,
                               terms=terms, device=device, eps_in=eps_in, eps_out=eps_out,
                               **defaults)
    self._last = None

  @property
  def batch(self) -> engine.Batch:
    return self._batch

  @property
  def n_atoms(self) -> int:
    return self._batch.n_atoms

  def _device_positions(self, r):
    """r as a contiguous float64 (n, 3) CUDA torch tensor when it is a CUDA
    array (a torch tensor or any DLPack producer), else None."""
    dev = getattr(r, "__dlpack_device__", None)
    if dev is None or dev()[0] != 2:  # 2: kDLCUDA
      return None
    import torch
    t = r if isinstance(r, torch.Tensor) else torch.from_dlpack(r)
    if t.device.index != self._batch.ctx.device:
      raise ValueError(f"positions on cuda:{t.device.index}, the energy function on "
                       f"cuda:{self._batch.ctx.device}")
    return t.detach().to(torch.float64).reshape(self.n_atoms, 3).contiguous()

  def _eval_device(self, t):
    """(energies (NTERMS,), forces (n, 3)) as CUDA tensors, computed on the
    caller's current stream without a host copy or synchronisation."""
    import torch
    e = torch.empty(len(TERM_NAMES), dtype=torch.float64, device=t.device)
    f = torch.empty_like(t)
    stream = torch.cuda.current_stream(t.device).cuda_stream
    self._batch.energy_forces_device(t.data_ptr(), e.data_ptr(), f.data_ptr(), stream)
    self._last = None  # the batch now holds these positions
    return e, f

  def _eval(self, r):
    t = self._device_positions(r)
    if t is not None:
      return self._eval_device(t)
    r = np.ascontiguousarray(np.asarray(r, dtype=np.float64).reshape(self.n_atoms, 3))
    if self._last is not None and np.array_equal(self._last[0], r):
      return self._last[1], self._last[2]
    self._batch.set_positions(r)
    e, f = self._batch.energy_forces()
    self._last = (r.copy(), e[0], f)
    return e[0], f

  def terms(self, r) -> dict:
    e, _ = self._eval(r)
    return {name: float(e[i]) for i, name in enumerate(TERM_NAMES)}

  def __call__(self, r, neighbor=None, **kwargs):
    """Total energy: a float, or a 0-d CUDA tensor when r is a CUDA array."""
    e = self._eval(r)[0][-1]
    return e if hasattr(e, "device") else float(e)

  def forces(self, r, neighbor=None, **kwargs):
    """-dE/dr (n, 3): NumPy, or a CUDA tensor when r is a CUDA array."""
    f = self._eval(r)[1]
    return f if hasattr(f, "device") else f.copy()

  def energy_and_forces(self, r, neighbor=None, **kwargs):
    e, f = self._eval(r)
    if hasattr(f, "device"):
      return e[-1], f
    return float(e[-1]), f.copy()

  def close(self):
    """Release the device batch now rather than at garbage collection."""
    self._batch.close()
    self._last = None

  def born_radii(self, r):
    t = self._device_positions(r)
    if t is not None:
      r = t.cpu().numpy()
    r = np.asarray(r, dtype=np.float64).reshape(self.n_atoms, 3)
    self._batch.set_positions(r)
    self._last = None
    return self._batch.born_radii()


def make_energy_fn(displacement_fn, system, cutoff_distance: float = 9.0,
                   return_decomposed: bool = False, implicit_solvent: bool = False,
                   exclusion_spec=None, **kwargs):
  """prolix ``make_energy_fn`` for ``implicit_solvent=True`` on the B200."""
  if not implicit_solvent:
    raise NotImplementedError(
        "prolix_b200 implements the implicit-solvent path only (implicit_solvent=True)")
  if kwargs.get("use_pbc", False):
    raise NotImplementedError("prolix_b200 implements free-space implicit solvent only "
                              "(use_pbc=True selects the reference's PME path)")
  sysd = system_to_dict(system)
  n = int(np.asarray(sysd["charges"]).shape[0])
  if n == 0:
    raise ValueError("make_energy_fn: system['charges'] is empty — cannot infer n_atoms")
  if "positions" not in sysd:
    sysd["positions"] = kwargs.get("positions", np.zeros((n, 3)))
  if "radii" not in sysd or sysd["radii"] is None:
    sysd["radii"] = np.ones(n)
  if "scaled_radii" not in sysd or sysd["scaled_radii"] is None:
    sysd["scaled_radii"] = np.asarray(sysd["radii"])
  has_table = sysd.get("excl_indices") is not None and np.asarray(sysd["excl_indices"]).size > 0
  if exclusion_spec is not None and "excl_pairs" not in sysd and not has_table:
    # the spec is used only when the system has no table of its own (system.py:161-162)
    pairs, kind, lj14, c14 = _exclusions_from_spec(exclusion_spec, n)
    sysd["excl_pairs"], sysd["excl_kind"] = pairs, kind
    sysd["lj14_scale"], sysd["coul14_scale"] = lj14, c14
  elif "excl_pairs" not in sysd and not has_table:
    # no spec and no table: the reference's (N, 0) table excludes nothing
    sysd["excl_pairs"] = np.zeros((0, 2), np.int32)
    sysd["excl_kind"] = np.zeros(0, np.int32)
  if exclusion_spec is not None and "exception_pairs" not in sysd:
    # explicit 1-4 overrides (system.py:149-159): their own energy term
    for k in ("exception_pairs", "exception_sigmas", "exception_epsilons", "exception_chargeprods"):
      v = getattr(exclusion_spec, k, None)
      if v is not None:
        sysd[k] = np.asarray(v)
  cutoff = float(kwargs.get("cutoff", cutoff_distance))
  eps_in = float(kwargs.get("solute_dielectric", 1.0))
  eps_out = float(kwargs.get("solvent_dielectric", 78.5))
  fn = EnergyFn(sysd, cutoff if cutoff > 0 else 0.0, eps_in=eps_in, eps_out=eps_out,
                gb_cutoff=float(kwargs.get("gb_cutoff", 0.0)),
                born_cutoff=float(kwargs.get("born_cutoff", 0.0)),
                device=int(kwargs.get("device", 0)))
  if not return_decomposed:
    return fn

  def term(name):
    return lambda r, n=None: fn.terms(r)[name]

  def electrostatics(r, neighbor=None):
    t = fn.terms(r)
    return t["gb"], t["coulomb"], fn.born_radii(r)

  def nonpolar(r, born_radii=None):
    return fn.terms(r)["nonpolar"]

  return {
      "bond": term("bond"), "angle": term("angle"), "dihedral": term("dihedral"),
      "improper": term("improper"), "urey_bradley": term("urey_bradley"), "cmap": term("cmap"),
      "lj": term("lj"),
      "exception": term("exception"), "electrostatics": electrostatics, "nonpolar": nonpolar,
      "total": fn,
  }
