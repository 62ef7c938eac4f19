"""ctypes binding of the C ABI declared in include/prolix_b200.h.

The CUDA library is required: there is no CPU fallback, and loading fails
loudly when ``libprolix_b200.so`` is missing or no sm_100 device is present.
``PROLIX_B200_LIB`` overrides the library path (an alternative build).
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

from . import _build

PB2_OK = 0
ERRORS = {
    -1: "invalid argument", -2: "out of memory", -3: "CUDA error",
    -4: "neighbour-list overflow", -5: "non-finite values", -6: "device wait timed out",
    -7: "no usable sm_100 device",
}

TERM_NAMES = ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar", "exception",
              "improper", "urey_bradley", "total")
NTERMS = 12
ABI_VERSION = 3  # PB2_ABI_VERSION of the structures mirrored below
USE_BONDED, USE_CMAP, USE_LJ, USE_COULOMB, USE_GB = 0x1, 0x2, 0x4, 0x8, 0x10
USE_ALL = 0x1F
FUSE_BONDED, FUSE_FINALIZE = 0x1, 0x2
STATUS_NONFINITE, STATUS_NLOVERFLOW, STATUS_FORCE_RANGE, STATUS_WAIT_TIMEOUT = 0x1, 0x2, 0x4, 0x8

_c_dp = ctypes.POINTER(ctypes.c_double)
_c_ip = ctypes.POINTER(ctypes.c_int32)


class SystemDesc(ctypes.Structure):
  _fields_ = [
      ("n_atoms", ctypes.c_int32),
      ("positions", _c_dp), ("charges", _c_dp), ("sigmas", _c_dp), ("epsilons", _c_dp),
      ("radii", _c_dp), ("scaled_radii", _c_dp), ("masses", _c_dp),
      ("n_bonds", ctypes.c_int32), ("bonds", _c_ip), ("bond_params", _c_dp),
      ("n_angles", ctypes.c_int32), ("angles", _c_ip), ("angle_params", _c_dp),
      ("n_torsions", ctypes.c_int32), ("n_torsion_terms", ctypes.c_int32),
      ("torsions", _c_ip), ("torsion_params", _c_dp),
      ("n_cmap", ctypes.c_int32), ("cmap_rows", _c_ip), ("cmap_map", _c_ip),
      ("n_cmap_maps", ctypes.c_int32), ("cmap_grid", ctypes.c_int32), ("cmap_coeffs", _c_dp),
      ("n_excl", ctypes.c_int32), ("excl_pairs", _c_ip), ("excl_kind", _c_ip),
      ("lj14_scale", ctypes.c_double), ("coul14_scale", ctypes.c_double),
      ("eps_in", ctypes.c_double), ("eps_out", ctypes.c_double),
      ("k_gb", ctypes.c_double), ("k_coulomb", ctypes.c_double),
      ("key", ctypes.c_uint32 * 2),
      ("dt", ctypes.c_double), ("kT", ctypes.c_double), ("gamma", ctypes.c_double),
      ("use_origin", ctypes.c_int32), ("origin", ctypes.c_double * 3),
      ("n_exceptions", ctypes.c_int32), ("exception_pairs", _c_ip), ("exception_params", _c_dp),
      ("n_impropers", ctypes.c_int32), ("n_improper_terms", ctypes.c_int32),
      ("improper_form", ctypes.c_int32), ("impropers", _c_ip), ("improper_params", _c_dp),
      ("n_urey_bradley", ctypes.c_int32), ("urey_bradley_bonds", _c_ip),
      ("urey_bradley_params", _c_dp),
  ]


class RunParams(ctypes.Structure):
  _fields_ = [
      ("terms", ctypes.c_uint32),
      ("cutoff", ctypes.c_double),
      ("skin", ctypes.c_double),
      ("nl_capacity", ctypes.c_int32),
      ("tile_segment", ctypes.c_int32),
      ("graph_chunk", ctypes.c_int32),
      ("partitionable_keys", ctypes.c_int32),
      ("gb_cutoff", ctypes.c_double),
      ("born_cutoff", ctypes.c_double),
      ("keep_atom_order", ctypes.c_int32),
      ("pair_list", ctypes.c_int32),
  ]


# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("pb2_abi_version", ctypes.c_int, []),
    ("pb2_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("pb2_ctx_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("pb2_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("pb2_batch_create", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(SystemDesc),
                                        ctypes.POINTER(RunParams), ctypes.POINTER(ctypes.c_void_p)]),
    ("pb2_batch_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("pb2_batch_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_int64)]),
    ("pb2_energy_forces", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    ("pb2_born_radii", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_set_positions", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_langevin_init", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_langevin_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("pb2_get_state", ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 6),
    ("pb2_set_state", ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4),
    ("pb2_set_full_state", ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 5),
    ("pb2_langevin_run_host", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_langevin_run_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("pb2_min_setup", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_min_sd", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    ("pb2_min_fire", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int32, ctypes.c_void_p]),
    ("pb2_min_rms", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_min_lbfgs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_permute_systems", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_energy_forces_device", ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4),
    ("pb2_traj_setup", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("pb2_traj_snapshot", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("pb2_traj_fetch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32] + [ctypes.c_void_p] * 4),
    ("pb2_get_status", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p]),
    ("pb2_langevin_center_momentum", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_set_langevin_params", ctypes.c_int, [ctypes.c_void_p] * 5),
    ("pb2_set_safeguards", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double]),
    ("pb2_get_safeguards", ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_double)] * 3),
    ("pb2_get_warn_counts", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p]),
    ("pb2_nl_build", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_nl_check", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p]),
    ("pb2_nl_capacity", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("pb2_nl_get", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_nl_last_build_ms", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("pb2_set_tile_segment", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("pb2_get_tile_segment", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("pb2_retire_system", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("pb2_test_hold_system", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    ("pb2_block_shapes", ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    ("pb2_set_block_shape", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("pb2_get_block_shape", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    ("pb2_set_force_blocks", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("pb2_get_force_blocks", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("pb2_set_fusion", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("pb2_get_fusion", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("pb2_set_profiling", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("pb2_last_timings", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("pb2_fp32_peak", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("pb2_diag_div_check", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_ulonglong,
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]),
    ("pb2_born_radii_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                              ctypes.c_void_p, ctypes.c_void_p]),
]

_LOCK = threading.Lock()
_LIB = None


def load(path=None) -> ctypes.CDLL:
  """Load the CUDA library (building it in-tree first if it is absent)."""
  global _LIB
  with _LOCK:
    if _LIB is None:
      env = os.environ.get("PROLIX_B200_LIB")
      p = Path(path or env or _build.CUDA_LIB)
      if not p.exists():
        _build.build_cuda()
      lib = ctypes.CDLL(str(p))
      for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
      if lib.pb2_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{p}: ABI version {lib.pb2_abi_version()}, this package needs "
                           f"{ABI_VERSION}; rebuild the library")
      _LIB = lib
  return _LIB


class PB2Error(RuntimeError):
  def __init__(self, code, msg):
    super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
    self.code = code
