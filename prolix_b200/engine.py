"""Device-resident ragged batch of implicit-solvent systems (host wrapper of
the C ABI).

A ``Batch`` holds any number of systems of any sizes; one force evaluation
or one Langevin step advances all of them with one launch per kernel.
"""

from __future__ import annotations

import ctypes
import math
import threading

import numpy as np

from . import _lib, topology

AKMA_TIME_FS = 48.88821291839  # prolix simulate.py:56
KB_KCAL = 0.0019872041          # prolix simulate.py:57
# the limits of prolix's batched Langevin step (batched_simulate.py:269, 290, 338)
BATCHED_SAFEGUARDS = {"vlimit": 20.0, "max_dx": 0.5, "force_cap": 1e4}
WARN_VLIMIT, WARN_FORCE_CAP, WARN_CONSTR_VIOL, WARN_DX_CAP = 0, 1, 2, 3  # typing.py:559-562
K_COULOMB = 332.0637            # prolix physics/system.py:135


def akma_dt(dt_fs: float) -> float:
  return dt_fs / AKMA_TIME_FS


def akma_gamma(gamma_per_ps: float) -> float:
  return gamma_per_ps * AKMA_TIME_FS * 1e-3


class Context:
  """One CUDA device.  Contexts are shared per device within a process."""

  _cache: dict[int, "Context"] = {}
  _lock = threading.Lock()

  def __init__(self, device: int = 0):
    self.lib = _lib.load()
    h = ctypes.c_void_p()
    rc = self.lib.pb2_ctx_create(int(device), ctypes.byref(h))
    if rc != _lib.PB2_OK:
      raise _lib.PB2Error(rc, f"cannot open device {device} (an sm_100 GPU is required)")
    self.handle = h
    self.device = device

  @classmethod
  def get(cls, device: int = 0) -> "Context":
    with cls._lock:
      if device not in cls._cache:
        cls._cache[device] = Context(device)
      return cls._cache[device]

  def check(self, rc: int):
    if rc != _lib.PB2_OK:
      msg = self.lib.pb2_last_error(self.handle)
      raise _lib.PB2Error(rc, msg.decode() if msg else "")


def _f64(a, shape=None):
  a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
  if shape is not None:
    a = a.reshape(shape)
  return a


def _i32(a, shape=None):
  a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
  if shape is not None:
    a = a.reshape(shape)
  return a


def _dp(a):
  return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
  return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _first(system, *keys):
  """The first of ``keys`` that holds a non-empty array (the fallback order
  of make_energy_fn, system.py:60-76), else None."""
  for k in keys:
    v = system.get(k)
    if v is not None and np.asarray(v).size:
      return v
  return None


def prepare_system(system: dict, *, dt=None, kT=None, gamma=None, key=None, eps_in=1.0,
                   eps_out=78.5, k_gb=K_COULOMB, k_coulomb=K_COULOMB,
                   lj14=topology.LJ14_DEFAULT, coul14=topology.COUL14_DEFAULT):
  """Normalise a system dict into the arrays of one ``pb2_system_desc``."""
  pos = _f64(system["positions"])
  n = pos.reshape(-1, 3).shape[0]
  pos = pos.reshape(n, 3)
  out = {"n": n, "positions": pos}
  for k in ("charges", "sigmas", "epsilons", "radii", "scaled_radii", "masses"):
    if k not in system and k == "masses":
      out[k] = np.ones(n)
      continue
    out[k] = _f64(system[k], (n,))
  bonds = _i32(system.get("bonds", np.zeros((0, 2))), (-1, 2))
  out["bonds"] = bonds
  out["bond_params"] = _f64(system.get("bond_params", np.zeros((0, 2))), (-1, 2))
  out["angles"] = _i32(system.get("angles", np.zeros((0, 3))), (-1, 3))
  out["angle_params"] = _f64(system.get("angle_params", np.zeros((0, 2))), (-1, 2))
  dih = _first(system, "dihedrals", "proper_dihedrals")
  dih = _i32(np.zeros((0, 4)) if dih is None else dih, (-1, 4))
  dp = _first(system, "dihedral_params", "proper_dihedral_params")
  dp = np.zeros((0, 1, 3)) if dp is None else np.asarray(dp, dtype=np.float64)
  if dp.ndim == 2:
    dp = dp[:, None, :]
  out["dihedrals"] = dih
  out["dihedral_params"] = _f64(dp).reshape(dih.shape[0], -1, 3) if dih.shape[0] else np.zeros((0, 1, 3))
  # impropers: the parameters' last axis picks the form as system.py:77-83 does
  # (2: harmonic (k, phi0), else periodic (n, phase, k))
  imp = _first(system, "impropers", "improper_dihedrals")
  imp = _i32(np.zeros((0, 4)) if imp is None else imp, (-1, 4))
  ipar = _first(system, "improper_params", "improper_dihedral_params")
  if imp.shape[0]:
    if ipar is None:
      raise ValueError("impropers given without improper_params")
    ipar = np.asarray(ipar, dtype=np.float64)
    if ipar.ndim == 2:
      ipar = ipar[:, None, :]
    width = ipar.shape[-1]
    if width not in (2, 3):
      raise ValueError(f"improper_params rows must be (k, phi0) or (n, phase, k), got {width} values")
    out["improper_form"] = 1 if width == 2 else 0
    out["improper_params"] = _f64(ipar).reshape(imp.shape[0], -1, width)
  else:
    out["improper_form"] = 0
    out["improper_params"] = np.zeros((0, 1, 3))
  out["impropers"] = imp
  ub = _first(system, "urey_bradley_bonds")
  out["urey_bradley_bonds"] = _i32(np.zeros((0, 2)) if ub is None else ub, (-1, 2))
  ubp = _first(system, "urey_bradley_params")
  if out["urey_bradley_bonds"].shape[0] and ubp is None:
    raise ValueError("urey_bradley_bonds given without urey_bradley_params")
  out["urey_bradley_params"] = _f64(np.zeros((0, 2)) if ubp is None else ubp, (-1, 2))
  if "cmap_torsions" in system and len(system["cmap_torsions"]):
    grids = np.asarray(system["cmap_energy_grids"], dtype=np.float64)
    if grids.ndim == 2:
      grids = grids[None]
    out["cmap_rows"] = _i32(system["cmap_torsions"], (-1, 5))
    out["cmap_map"] = _i32(system.get("cmap_indices", np.zeros(out["cmap_rows"].shape[0])))
    out["cmap_coeffs"] = _f64(np.stack([topology.cmap_coefficients(g) for g in grids]))
    out["cmap_grid"] = grids.shape[1]
  else:
    out["cmap_rows"] = np.zeros((0, 5), np.int32)
    out["cmap_map"] = np.zeros(0, np.int32)
    out["cmap_coeffs"] = np.zeros((1, 1, 1, 16))
    out["cmap_grid"] = 1
  if "excl_pairs" in system:
    out["excl_pairs"] = _i32(system["excl_pairs"], (-1, 2))
    out["excl_kind"] = _i32(system["excl_kind"])
  elif system.get("excl_indices") is not None:
    # prolix's per-atom padded table (map_exclusions_to_dense_padded)
    pairs, kind, t_lj14, t_c14 = topology.pairs_from_padded_table(
        system["excl_indices"], system.get("excl_scales_vdw"), system.get("excl_scales_elec"))
    out["excl_pairs"], out["excl_kind"] = pairs, kind
    lj14 = system.get("lj14_scale", t_lj14)
    coul14 = system.get("coul14_scale", t_c14)
  else:
    out["excl_pairs"], out["excl_kind"] = topology.exclusion_pairs(bonds, n)
  out["scal"] = dict(lj14=float(system.get("lj14_scale", lj14)),
                     coul14=float(system.get("coul14_scale", coul14)),
                     eps_in=float(system.get("solute_dielectric", eps_in)),
                     eps_out=float(system.get("solvent_dielectric", eps_out)),
                     k_gb=float(k_gb), k_coulomb=float(k_coulomb))
  k = system.get("key", key)
  if k is None:
    k = (0, int(system.get("seed", 0)) & 0xFFFFFFFF)
  out["key"] = tuple(int(v) & 0xFFFFFFFF for v in np.asarray(k).reshape(2))
  out["dt"] = float(system.get("dt", dt if dt is not None else akma_dt(1.0)))
  out["kT"] = float(system.get("kT", kT if kT is not None else 300.0 * KB_KCAL))
  out["gamma"] = float(system.get("gamma", gamma if gamma is not None else akma_gamma(1.0)))
  out["origin"] = None if system.get("origin") is None else tuple(float(v) for v in system["origin"])
  # explicit 1-4 exception pairs, ExclusionSpec field names (neighbor_list.py:44-50)
  ep = system.get("exception_pairs")
  if ep is not None and np.asarray(ep).size:
    out["exception_pairs"] = _i32(ep, (-1, 2))
    m = out["exception_pairs"].shape[0]
    out["exception_params"] = _f64(np.stack([
        np.asarray(system["exception_chargeprods"], dtype=np.float64).reshape(m),
        np.asarray(system["exception_sigmas"], dtype=np.float64).reshape(m),
        np.asarray(system["exception_epsilons"], dtype=np.float64).reshape(m)], axis=1))
  else:
    out["exception_pairs"] = np.zeros((0, 2), np.int32)
    out["exception_params"] = np.zeros((0, 3))
  return out


def default_origin(positions) -> tuple:
  """The origin a batch picks for a system: its rounded centroid (A)."""
  c = np.asarray(positions, dtype=np.float64).reshape(-1, 3).mean(axis=0)
  return tuple(float(v) for v in np.round(c))


def _desc(p) -> _lib.SystemDesc:
  d = _lib.SystemDesc()
  d.n_atoms = p["n"]
  d.positions = _dp(p["positions"])
  for k in ("charges", "sigmas", "epsilons", "radii", "scaled_radii", "masses"):
    setattr(d, k, _dp(p[k]))
  d.n_bonds = p["bonds"].shape[0]
  d.bonds, d.bond_params = _ip(p["bonds"]), _dp(p["bond_params"])
  d.n_angles = p["angles"].shape[0]
  d.angles, d.angle_params = _ip(p["angles"]), _dp(p["angle_params"])
  d.n_torsions = p["dihedrals"].shape[0]
  d.n_torsion_terms = p["dihedral_params"].shape[1] if d.n_torsions else 1
  d.torsions, d.torsion_params = _ip(p["dihedrals"]), _dp(p["dihedral_params"])
  d.n_cmap = p["cmap_rows"].shape[0]
  d.cmap_rows, d.cmap_map = _ip(p["cmap_rows"]), _ip(p["cmap_map"])
  d.n_cmap_maps = p["cmap_coeffs"].shape[0]
  d.cmap_grid = p["cmap_grid"]
  d.cmap_coeffs = _dp(p["cmap_coeffs"])
  d.n_excl = p["excl_pairs"].shape[0]
  d.excl_pairs, d.excl_kind = _ip(p["excl_pairs"]), _ip(p["excl_kind"])
  s = p["scal"]
  d.lj14_scale, d.coul14_scale = s["lj14"], s["coul14"]
  d.eps_in, d.eps_out = s["eps_in"], s["eps_out"]
  d.k_gb, d.k_coulomb = s["k_gb"], s["k_coulomb"]
  d.key[0], d.key[1] = p["key"]
  d.dt, d.kT, d.gamma = p["dt"], p["kT"], p["gamma"]
  if p["origin"] is not None:
    d.use_origin = 1
    d.origin[0], d.origin[1], d.origin[2] = p["origin"]
  d.n_exceptions = p["exception_pairs"].shape[0]
  d.exception_pairs, d.exception_params = _ip(p["exception_pairs"]), _dp(p["exception_params"])
  d.n_impropers = p["impropers"].shape[0]
  d.n_improper_terms = p["improper_params"].shape[1] if d.n_impropers else 1
  d.improper_form = p["improper_form"]
  d.impropers, d.improper_params = _ip(p["impropers"]), _dp(p["improper_params"])
  d.n_urey_bradley = p["urey_bradley_bonds"].shape[0]
  d.urey_bradley_bonds = _ip(p["urey_bradley_bonds"])
  d.urey_bradley_params = _dp(p["urey_bradley_params"])
  return d


class Batch:
  """A ragged batch of systems resident on one GPU."""

  def __init__(self, systems, *, cutoff=0.0, gb_cutoff=-1.0, born_cutoff=0.0, skin=2.0, terms=_lib.USE_ALL,
               device=0,
               tile_segment=0, graph_chunk=50, partitionable_keys=True, nl_capacity=0,
               keep_atom_order=False, pair_list=True, **system_defaults):
    if isinstance(systems, dict):
      systems = [systems]
    if not systems:
      raise ValueError("a batch needs at least one system")
    self.ctx = Context.get(device)
    self.lib = self.ctx.lib
    self.prepared = [prepare_system(s, **system_defaults) for s in systems]
    self.sizes = np.array([p["n"] for p in self.prepared], dtype=np.int64)
    self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
    self.n_systems = len(self.prepared)
    self.n_atoms = int(self.offsets[-1])
    self.cutoff = float(cutoff)
    descs = (_lib.SystemDesc * self.n_systems)(*[_desc(p) for p in self.prepared])
    rp = _lib.RunParams(terms=int(terms), cutoff=float(cutoff), skin=float(skin),
                        nl_capacity=int(nl_capacity), tile_segment=int(tile_segment),
                        graph_chunk=int(graph_chunk),
                        partitionable_keys=1 if partitionable_keys else 0,
                        gb_cutoff=float(gb_cutoff), born_cutoff=float(born_cutoff),
                        keep_atom_order=1 if keep_atom_order else 0,
                        pair_list=0 if pair_list else -1)
    h = ctypes.c_void_p()
    self.ctx.check(self.lib.pb2_batch_create(self.ctx.handle, self.n_systems, descs,
                                             ctypes.byref(rp), ctypes.byref(h)))
    self.handle = h
    self._stream = None

  # ---------------------------------------------------------------- helpers
  def _check(self, rc):
    self.ctx.check(rc)

  def split(self, flat):
    """Split a batch-order (n_atoms, ...) array into per-system arrays."""
    return [flat[self.offsets[s]:self.offsets[s + 1]] for s in range(self.n_systems)]

  def close(self):
    if getattr(self, "handle", None):
      self.lib.pb2_batch_destroy(self.handle)
      self.handle = None

  def __del__(self):
    try:
      self.close()
    except Exception:
      pass

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()

  # ---------------------------------------------------------------- physics
  def energy_forces(self, stream=None):
    """(energies (n_systems, NTERMS) with columns TERM_NAMES, forces (n_atoms, 3))."""
    e = np.zeros((self.n_systems, _lib.NTERMS))
    f = np.zeros((self.n_atoms, 3))
    self._check(self.lib.pb2_energy_forces(self.handle, e.ctypes.data, f.ctypes.data, stream))
    return e, f

  def forces(self, stream=None):
    f = np.zeros((self.n_atoms, 3))
    self._check(self.lib.pb2_energy_forces(self.handle, None, f.ctypes.data, stream))
    return f

  def born_radii(self, stream=None):
    b = np.zeros(self.n_atoms)
    self._check(self.lib.pb2_born_radii(self.handle, b.ctypes.data, stream))
    return b

  def set_positions(self, positions, stream=None):
    x = _f64(positions, (self.n_atoms, 3))
    self._check(self.lib.pb2_set_positions(self.handle, x.ctypes.data, stream))

  def langevin_init(self, stream=None):
    self._check(self.lib.pb2_langevin_init(self.handle, stream))

  def langevin_run(self, n_steps, stream=None):
    self._check(self.lib.pb2_langevin_run(self.handle, int(n_steps), stream))

  def get_state(self, stream=None, fields=("position", "momentum", "force", "key", "step"),
                out=None):
    """Read the BAOAB state.  ``fields`` selects what is copied; ``out`` may
    supply destination arrays by field name (C-contiguous, float64 (n, 3) for
    position/momentum/force), e.g. page-locked buffers for full-speed copies."""
    out = dict(out or {})
    shapes = {"position": ((self.n_atoms, 3), np.float64), "momentum": ((self.n_atoms, 3), np.float64),
              "force": ((self.n_atoms, 3), np.float64), "key": ((self.n_systems, 2), np.uint32),
              "step": ((self.n_systems,), np.int64)}
    res = {}
    for name in fields:
      shape, dt = shapes[name]
      a = out.get(name)
      if a is None:
        a = np.zeros(shape, dtype=dt)
      elif a.shape != shape or a.dtype != dt or not a.flags.c_contiguous:
        raise ValueError(f"get_state: out[{name!r}] must be a C-contiguous {dt.__name__} {shape}")
      res[name] = a
    ptr = lambda name: res[name].ctypes.data if name in res else None
    self._check(self.lib.pb2_get_state(self.handle, ptr("position"), ptr("momentum"), ptr("force"),
                                       ptr("key"), ptr("step"), stream))
    return res

  def set_full_state(self, position, momentum, force, key=None, stream=None):
    """Restore x, p, F (and optionally the keys) without a force evaluation;
    ``force`` must be the forces at ``position`` as get_state returned them."""
    x = _f64(position, (self.n_atoms, 3))
    p = _f64(momentum, (self.n_atoms, 3))
    f = _f64(force, (self.n_atoms, 3))
    k = None if key is None else np.ascontiguousarray(np.asarray(key, dtype=np.uint32).reshape(-1, 2))
    self._check(self.lib.pb2_set_full_state(self.handle, x.ctypes.data, p.ctypes.data, f.ctypes.data,
                                            None if k is None else k.ctypes.data, stream))

  def langevin_run_host(self, position, momentum, force, n_steps, stream=None, copy_in=None, copy_out=None):
    """pb2_langevin_run_host: step the state held in the three (n_atoms, 3)
    float64 arrays and write the new state back into them.  Asynchronous:
    copies in on ``copy_in``, steps on ``stream``, copies out on
    ``copy_out`` (each defaults to ``stream``); the arrays must stay alive
    and untouched until ``copy_out`` has finished.  Page-locked arrays let
    the copies overlap other streams' work."""
    copy_in = stream if copy_in is None else copy_in
    copy_out = stream if copy_out is None else copy_out
    arrs = (position, momentum, force)
    for a in arrs:
      if (not isinstance(a, np.ndarray) or a.shape != (self.n_atoms, 3) or a.dtype != np.float64
          or not a.flags.c_contiguous or not a.flags.writeable):
        raise ValueError(f"langevin_run_host: arrays must be writeable C-contiguous float64 ({self.n_atoms}, 3)")
    self._check(self.lib.pb2_langevin_run_host(self.handle, position.ctypes.data, momentum.ctypes.data,
                                               force.ctypes.data, int(n_steps), stream, copy_in, copy_out))

  def langevin_run_device(self, position_ptr, momentum_ptr, force_ptr, n_steps, stream=None):
    """pb2_langevin_run_device: the functional step on caller-owned device
    arrays ((n_atoms, 3) float64 row-major, e.g. torch tensors'
    data_ptr()), overwritten with the new state; asynchronous on
    ``stream``."""
    if not (position_ptr and momentum_ptr and force_ptr):
      raise ValueError("langevin_run_device: three device pointers are required")
    self._check(self.lib.pb2_langevin_run_device(self.handle, position_ptr, momentum_ptr, force_ptr,
                                                 int(n_steps), stream))

  def energy_forces_device(self, positions_ptr, energies_ptr, forces_ptr, stream=None):
    """pb2_energy_forces_device on raw device pointers (e.g. a torch tensor's
    data_ptr()); any may be 0/None.  Asynchronous on ``stream``."""
    self._check(self.lib.pb2_energy_forces_device(self.handle, positions_ptr or None, energies_ptr or None,
                                                  forces_ptr or None, stream))

  # --------------------------------------------------------- trajectory ring
  def traj_setup(self, capacity: int):
    self._check(self.lib.pb2_traj_setup(self.handle, int(capacity)))
    self.traj_capacity = int(capacity)

  def traj_snapshot(self, slot: int, stream=None):
    self._check(self.lib.pb2_traj_snapshot(self.handle, int(slot), stream))

  def traj_fetch(self, first: int, count: int, stream=None):
    """(positions (count, n_atoms, 3) float32, velocities, steps (count, n_systems))."""
    pos = np.empty((count, self.n_atoms, 3), np.float32)
    vel = np.empty((count, self.n_atoms, 3), np.float32)
    steps = np.empty((count, self.n_systems), np.int64)
    self._check(self.lib.pb2_traj_fetch(self.handle, int(first), int(count), pos.ctypes.data,
                                        vel.ctypes.data, steps.ctypes.data, stream))
    return pos, vel, steps

  def permute_systems(self, perm, stream=None):
    """Slot s takes x, p and F of slot perm[s] (replica exchange); keys,
    step counters, kT and dt stay with the slots."""
    pm = np.ascontiguousarray(np.asarray(perm, dtype=np.int32).reshape(self.n_systems))
    self._check(self.lib.pb2_permute_systems(self.handle, pm.ctypes.data, stream))

  # ------------------------------------------------------------ minimiser
  def min_setup(self, heavy=None, backbone=None):
    """Take the current positions as the restraint reference; per-atom
    heavy / backbone selections (batch order), default mass > 1.1 amu."""
    def mask(m):
      if m is None:
        return None
      return np.ascontiguousarray(np.asarray(m, dtype=np.uint8).reshape(self.n_atoms))
    h, bb = mask(heavy), mask(backbone)
    self._min_masks = (h, bb)  # keep alive for the call
    self._check(self.lib.pb2_min_setup(self.handle, None if h is None else h.ctypes.data,
                                       None if bb is None else bb.ctypes.data))

  MIN_KIND = {"all": 0, "heavy": 1, "backbone": 2}

  def min_sd(self, n_steps, k=0.0, kind="all", dt=0.002, max_dx=0.01, stream=None):
    self._check(self.lib.pb2_min_sd(self.handle, int(n_steps), float(k), self.MIN_KIND[kind],
                                    float(dt), float(max_dx), stream))

  def min_fire(self, n_steps, k=0.0, kind="all", dt_start=1e-4, dt_max=1e-3, max_disp=0.1, force_cap=0.0,
               keep_best=True, stream=None):
    """One FIRE stage; max_disp / force_cap 0 disable the caps; keep_best
    ends at the lowest-RMS positions (batched_minimize), else at the last."""
    self._check(self.lib.pb2_min_fire(self.handle, int(n_steps), float(k), self.MIN_KIND[kind],
                                      float(dt_start), float(dt_max), float(max_disp), float(force_cap),
                                      1 if keep_best else 0, stream))

  def min_lbfgs(self, n_iter, tol=1e-6, max_step=0.1, hist=10, max_trials=30, stream=None):
    """L-BFGS polish of every system; returns the per-system converged flags."""
    conv = np.zeros(self.n_systems, dtype=np.int32)
    self._check(self.lib.pb2_min_lbfgs(self.handle, int(n_iter), float(tol), float(max_step), int(hist),
                                       int(max_trials), conv.ctypes.data, stream))
    return conv.astype(bool)

  def min_rms(self, stream=None):
    """Per-system RMS over atoms of the unrestrained force, kcal/mol/A."""
    out = np.zeros(self.n_systems)
    self._check(self.lib.pb2_min_rms(self.handle, out.ctypes.data, stream))
    return out

  def set_state(self, position=None, momentum=None, key=None, stream=None):
    x = None if position is None else _f64(position, (self.n_atoms, 3))
    p = None if momentum is None else _f64(momentum, (self.n_atoms, 3))
    k = None if key is None else np.ascontiguousarray(np.asarray(key, dtype=np.uint32).reshape(-1, 2))
    self._check(self.lib.pb2_set_state(self.handle, None if x is None else x.ctypes.data,
                                       None if p is None else p.ctypes.data,
                                       None if k is None else k.ctypes.data, stream))

  def status(self, clear=False, stream=None):
    s = np.zeros(self.n_systems, dtype=np.uint32)
    self._check(self.lib.pb2_get_status(self.handle, s.ctypes.data, 1 if clear else 0, stream))
    return s

  def set_langevin_params(self, dt=None, kT=None, gamma=None, stream=None):
    """New dt (tau), kT (kcal/mol) and/or gamma (1/tau) for the following
    steps: a scalar for every system or one value per system; None keeps."""
    def arr(v):
      if v is None:
        return None
      return np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (self.n_systems,)))
    d, k, g = arr(dt), arr(kT), arr(gamma)
    self._check(self.lib.pb2_set_langevin_params(self.handle, None if d is None else d.ctypes.data,
                                                 None if k is None else k.ctypes.data,
                                                 None if g is None else g.ctypes.data, stream))

  def center_momentum(self, stream=None):
    """Subtract each system's mean momentum (jax_md center_velocity; a
    one-atom system is left alone)."""
    self._check(self.lib.pb2_langevin_center_momentum(self.handle, stream))

  def set_safeguards(self, vlimit=0.0, max_dx=0.0, force_cap=0.0):
    """Safeguards of prolix's batched Langevin step (batched_simulate.py:263-356):
    speed limit on |p/m| after the opening half kick, per-step displacement
    limit (A) and closing-force limit (kcal/mol/A); 0 turns each off.
    ``set_safeguards(**BATCHED_SAFEGUARDS)`` gives the reference's values."""
    self._check(self.lib.pb2_set_safeguards(self.handle, float(vlimit), float(max_dx),
                                            float(force_cap)))

  def safeguards(self) -> dict:
    v = [ctypes.c_double(0.0) for _ in range(3)]
    self._check(self.lib.pb2_get_safeguards(self.handle, *[ctypes.byref(x) for x in v]))
    return dict(zip(("vlimit", "max_dx", "force_cap"), (x.value for x in v)))

  def warn_counts(self, reset=False, stream=None):
    """(n_systems, 4) int32: steps in which each safeguard fired, columns in
    prolix's order (WARN_VLIMIT, WARN_FORCE_CAP, WARN_CONSTR_VIOL,
    WARN_DX_CAP; typing.py:559-563).  Column 1 is the reference's cap_count."""
    c = np.zeros((self.n_systems, 4), dtype=np.int32)
    self._check(self.lib.pb2_get_warn_counts(self.handle, c.ctypes.data, 1 if reset else 0, stream))
    return c

  def set_tile_segment(self, segment: int):
    self._check(self.lib.pb2_set_tile_segment(self.handle, int(segment)))

  def tile_segment(self) -> int:
    v = ctypes.c_int32(0)
    self._check(self.lib.pb2_get_tile_segment(self.handle, ctypes.byref(v)))
    return int(v.value)

  def retire(self, system: int, stream=None):
    """Stop stepping and evaluating one system (stream-ordered, irreversible):
    its state stays as the last step left it and it costs no more work."""
    self._check(self.lib.pb2_retire_system(self.handle, int(system), stream))

  def set_profiling(self, enable: bool):
    self._check(self.lib.pb2_set_profiling(self.handle, 1 if enable else 0))

  def last_timings(self):
    """Device ms of the last profiled run: born, finalize, force, chain,
    bonded, integrator, bounding boxes, whole run."""
    t = np.zeros(8)
    self._check(self.lib.pb2_last_timings(self.handle, t.ctypes.data))
    return t

  # neighbour list
  # ---------------------------------------------------------------- schedule
  def block_shapes(self, pass_: int) -> list:
    """(threads, min blocks per SM) compiled for pair pass 0 (descreening),
    1 (force), 2 (chain rule) or 3 (the force pass's four-block kernel)."""
    t = (ctypes.c_int32 * 8)()
    m = (ctypes.c_int32 * 8)()
    n = self.lib.pb2_block_shapes(int(pass_), t, m, 8)
    if n < 0:
      self._check(n)
    return [(int(t[k]), int(m[k])) for k in range(min(n, 8))]

  def set_block_shape(self, pass_: int, threads: int, min_blocks: int):
    self._check(self.lib.pb2_set_block_shape(self.handle, int(pass_), int(threads), int(min_blocks)))

  def block_shape(self, pass_: int) -> tuple:
    t, m = ctypes.c_int32(0), ctypes.c_int32(0)
    self._check(self.lib.pb2_get_block_shape(self.handle, int(pass_), ctypes.byref(t), ctypes.byref(m)))
    return int(t.value), int(m.value)

  def set_force_blocks(self, blocks: int):
    """I-blocks per warp of the force pass, 2 or 4 (the same forces bit for bit)."""
    self._check(self.lib.pb2_set_force_blocks(self.handle, int(blocks)))

  def force_blocks(self) -> int:
    v = ctypes.c_int32(0)
    self._check(self.lib.pb2_get_force_blocks(self.handle, ctypes.byref(v)))
    return int(v.value)

  def set_fusion(self, flags: int):
    """_lib.FUSE_* bits: the bonded terms in the chain pass, the Born-radius
    finalize in the descreening pass."""
    self._check(self.lib.pb2_set_fusion(self.handle, int(flags)))

  def fusion(self) -> int:
    f = ctypes.c_int32(0)
    self._check(self.lib.pb2_get_fusion(self.handle, ctypes.byref(f)))
    return int(f.value)

  def nl_build(self, stream=None):
    self._check(self.lib.pb2_nl_build(self.handle, stream))

  def nl_check(self, stream=None, wait=True):
    """Rebuild the neighbour list if an atom moved more than skin/2 since the
    last build.  wait=True: returns how many systems had; wait=False: only
    enqueues the check (and rebuild), returns None."""
    if not wait:
      self._check(self.lib.pb2_nl_check(self.handle, None, stream))
      return None
    r = ctypes.c_int32(0)
    self._check(self.lib.pb2_nl_check(self.handle, ctypes.byref(r), stream))
    return int(r.value)

  def nl_last_build_ms(self) -> float:
    """Device time of the last neighbour-list build (CUDA events)."""
    t = ctypes.c_double(0.0)
    self._check(self.lib.pb2_nl_last_build_ms(self.handle, ctypes.byref(t)))
    return float(t.value)

  def nl_capacity(self) -> int:
    c = ctypes.c_int32(0)
    self._check(self.lib.pb2_nl_capacity(self.handle, ctypes.byref(c)))
    return int(c.value)

  def nl_get(self, stream=None):
    k = self.nl_capacity()
    out = np.zeros((self.n_atoms, k), dtype=np.int32)
    self._check(self.lib.pb2_nl_get(self.handle, out.ctypes.data, stream))
    return out


def term_dict(row) -> dict:
  return {name: float(row[i]) for i, name in enumerate(_lib.TERM_NAMES)}
