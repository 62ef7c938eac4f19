"""ctypes wrapper of the C/OpenMP oracle (TEST INFRASTRUCTURE ONLY; see
oracle/c/oracle_forces.c for the formulas and their reference citations)."""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import cbuild, topology

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class _Sys(ctypes.Structure):
  _fields_ = [("n", ctypes.c_int), ("pos", _dp), ("q", _dp), ("sigma", _dp), ("eps", _dp),
              ("radii", _dp), ("sr", _dp), ("n_excl", ctypes.c_int), ("excl", _ip),
              ("excl_kind", _ip), ("lj14", ctypes.c_double), ("coul14", ctypes.c_double),
              ("eps_in", ctypes.c_double), ("eps_out", ctypes.c_double), ("k_gb", ctypes.c_double),
              ("k_coul", ctypes.c_double), ("cutoff", ctypes.c_double), ("gb_cutoff", ctypes.c_double),
              ("n_bond", ctypes.c_int), ("bond", _ip), ("bond_par", _dp),
              ("n_angle", ctypes.c_int), ("angle", _ip), ("angle_par", _dp),
              ("n_tors", ctypes.c_int), ("n_terms", ctypes.c_int), ("tors", _ip), ("tors_par", _dp)]


_LIB = None


def _lib():
  global _LIB
  if _LIB is None:
    lib = ctypes.CDLL(str(cbuild.build()))
    lib.pb2o_energy_forces.restype = ctypes.c_int
    lib.pb2o_energy_forces.argtypes = [ctypes.POINTER(_Sys), _dp, _dp, ctypes.c_int]
    _LIB = lib
  return _LIB


def _f(a, shape=None):
  a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
  return a.reshape(shape) if shape is not None else a


def _i(a, shape=None):
  a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
  return a.reshape(shape) if shape is not None else a


TERMS = ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar", "total")


def energy_forces(system, pos=None, cutoff=0.0, gb_cutoff=None, threads=0, eps_in=1.0,
                  eps_out=78.5, k=332.0637):
  """(energies dict, forces) in FP64; CMAP is not included (0), nor are
  explicit exclusion tables or exception pairs (the exclusions follow the
  bonds; ``exception`` is reported as 0)."""
  if "excl_pairs" in system or np.asarray(system.get("exception_pairs", np.zeros((0, 2)))).size:
    raise NotImplementedError("the C oracle derives exclusions from the bonds and has no exception pairs")
  pos = _f(system["positions"] if pos is None else pos, (-1, 3))
  n = pos.shape[0]
  pairs, sv, se = topology.pair_scales(system.get("bonds", np.zeros((0, 2))), n)
  kind = (sv != 0).astype(np.int32)
  keep = {}
  arrs = dict(pos=pos, q=_f(system["charges"]), sigma=_f(system["sigmas"]),
              eps=_f(system["epsilons"]), radii=_f(system["radii"]), sr=_f(system["scaled_radii"]),
              excl=_i(pairs, (-1, 2)), kind=_i(kind),
              bond=_i(system.get("bonds", np.zeros((0, 2))), (-1, 2)),
              bond_par=_f(system.get("bond_params", np.zeros((0, 2))), (-1, 2)),
              angle=_i(system.get("angles", np.zeros((0, 3))), (-1, 3)),
              angle_par=_f(system.get("angle_params", np.zeros((0, 2))), (-1, 2)),
              tors=_i(system.get("dihedrals", np.zeros((0, 4))), (-1, 4)))
  tp = np.asarray(system.get("dihedral_params", np.zeros((0, 1, 3))), dtype=np.float64)
  arrs["tors_par"] = _f(tp.reshape(arrs["tors"].shape[0], -1, 3)) if arrs["tors"].shape[0] else np.zeros((0, 1, 3))
  keep.update(arrs)
  s = _Sys(n=n, pos=arrs["pos"].ctypes.data_as(_dp), q=arrs["q"].ctypes.data_as(_dp),
           sigma=arrs["sigma"].ctypes.data_as(_dp), eps=arrs["eps"].ctypes.data_as(_dp),
           radii=arrs["radii"].ctypes.data_as(_dp), sr=arrs["sr"].ctypes.data_as(_dp),
           n_excl=arrs["excl"].shape[0], excl=arrs["excl"].ctypes.data_as(_ip),
           excl_kind=arrs["kind"].ctypes.data_as(_ip), lj14=topology.LJ14_SCALE,
           coul14=topology.COUL14_SCALE, eps_in=eps_in, eps_out=eps_out, k_gb=k, k_coul=k,
           cutoff=float(cutoff), gb_cutoff=-1.0 if gb_cutoff is None else float(gb_cutoff),
           n_bond=arrs["bond"].shape[0], bond=arrs["bond"].ctypes.data_as(_ip),
           bond_par=arrs["bond_par"].ctypes.data_as(_dp), n_angle=arrs["angle"].shape[0],
           angle=arrs["angle"].ctypes.data_as(_ip), angle_par=arrs["angle_par"].ctypes.data_as(_dp),
           n_tors=arrs["tors"].shape[0], n_terms=arrs["tors_par"].shape[1] if arrs["tors"].shape[0] else 1,
           tors=arrs["tors"].ctypes.data_as(_ip), tors_par=arrs["tors_par"].ctypes.data_as(_dp))
  e = np.zeros(9)
  f = np.zeros((n, 3))
  rc = _lib().pb2o_energy_forces(ctypes.byref(s), e.ctypes.data_as(_dp), f.ctypes.data_as(_dp),
                                 int(threads))
  if rc != 0:
    raise MemoryError("C oracle allocation failed")
  out = dict(zip(TERMS, e.tolist()))
  out["exception"] = 0.0
  return out, f


def threads() -> int:
  return os.cpu_count() or 1
