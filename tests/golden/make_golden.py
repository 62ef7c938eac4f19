"""Writes the golden fixtures of this directory.  Run from the repository
root: ``python tests/golden/make_golden.py``.

* ``known_answers.json``: the known answers the reference's own tests hold
  for this path, restated by hand with their sources, and published
  known-answer vectors of the third-party algorithms on it (threefry2x32,
  jax.random.split).  The reference cannot run here (JAX is not installed),
  so these are its only first-hand values.
* ``oracle_small.npz``: FP64 oracle outputs (per-term energies, forces,
  Born radii) for seeded small cases of the benchmark's shapes, and a
  zero-force BAOAB trajectory, frozen so that the oracle, the generator and
  the CUDA path are all checked against the same committed numbers.
"""

from __future__ import annotations

import hashlib
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

from oracle import energy, gbsa, integrator, prng, topology  # noqa: E402
from prolix_b200 import synth  # noqa: E402

K = gbsa.K_COULOMB
TAU = 1.0 / 1.0 - 1.0 / 78.5

KNOWN_ANSWERS = {
    "born_ion": {
        "source": "prolix tests/physics/test_generalized_born.py:11-52",
        "charge": 1.0, "radius": 2.0, "born_radius": 2.0 - 0.09,
        "gb_energy": -0.5 * K * TAU / (2.0 - 0.09), "gb_energy_rel": 1e-5,
    },
    "bond": {
        "source": "prolix tests/physics/test_bonded.py:10-30",
        "positions": [[0.0, 0.0, 0.0], [1.1, 0.0, 0.0]], "params": [1.0, 100.0],
        "energy": 0.5, "force_x": [10.0, -10.0], "force_abs": 1e-5,
    },
    "angle": {
        "source": "prolix tests/physics/test_bonded.py:32-59",
        "positions": [[1.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0]],
        "params": [math.pi, 100.0], "energy": 0.5 * 100.0 * (math.pi / 2) ** 2, "energy_rel": 1e-4,
    },
    "threefry2x32_20": {
        "source": "Random123 known-answer vectors (Salmon et al. 2011)",
        "cases": [[[0, 0], [0, 0], [0x6B200159, 0x99BA4EFE]],
                  [[0xFFFFFFFF, 0xFFFFFFFF], [0xFFFFFFFF, 0xFFFFFFFF], [0x1CB996FC, 0xBB002BE7]],
                  [[0x13198A2E, 0x03707344], [0x243F6A88, 0x85A308D3], [0xC4923A9C, 0x483DF7A0]]],
    },
    "jax_split_prngkey0": {
        "source": "jax.random.split(jax.random.PRNGKey(0)) as printed in JAX's documentation",
        "original": [[4146024105, 967050713], [2718843009, 1272950319]],
        "partitionable": [[1797259609, 2579123966], [928981903, 3453687069]],
    },
}

# (name, n_atoms, seed, compact, cmap, cutoff, explicit 1-4 exceptions)
CASES = [
    ("chain166_all_pairs", 166, 1, False, True, 0.0, False),
    ("globule600_cutoff20", 600, 600, True, True, 20.0, False),
    ("chain166_exceptions", 166, 2, True, False, 0.0, True),
]
ZERO_FORCE = ("chain97_zero_force", 97, 21, 1234, 7)  # name, n, seed, key seed, steps


def positions_digest(pos) -> str:
  return hashlib.sha256(np.ascontiguousarray(pos, dtype=np.float64).tobytes()).hexdigest()[:16]


def with_explicit_14(s):
  """The system with its 1-4 pairs excluded and restated as exception pairs
  carrying the scaled parameters (ExclusionSpec.from_protein layout)."""
  n = len(s["charges"])
  p12, p13, p14 = topology.bonded_pairs(s["bonds"], n)
  allp = np.sort(np.concatenate([p12, p13, p14]).astype(np.int64), axis=1)
  allp = allp[np.lexsort((allp[:, 1], allp[:, 0]))]
  q, sig, eps = (np.asarray(s[k], np.float64) for k in ("charges", "sigmas", "epsilons"))
  i, j = p14[:, 0], p14[:, 1]
  return dict(s, excl_pairs=allp.astype(np.int32), excl_kind=np.zeros(len(allp), np.int32),
              exception_pairs=p14.astype(np.int32),
              exception_chargeprods=q[i] * q[j] * topology.COUL14_SCALE,
              exception_sigmas=0.5 * (sig[i] + sig[j]) * 1.05,
              exception_epsilons=topology.LJ14_SCALE * np.sqrt(eps[i] * eps[j]))


def case_system(name):
  for c in CASES:
    if c[0] == name:
      _, n, seed, compact, cmap, cutoff, exc = c
      s = synth.make_chain(n, seed, compact=compact, cmap=cmap)
      return (with_explicit_14(s) if exc else s), cutoff
  raise KeyError(name)


def zero_force_run():
  name, n, seed, kseed, steps = ZERO_FORCE
  s = synth.make_chain(n, seed, compact=True)
  dt, kT, gamma = integrator.akma_dt(1.0), integrator.kT_of(300.0), integrator.akma_gamma(1.0)
  zero = lambda r: np.zeros_like(r)
  st = integrator.init(zero, prng.prng_key(kseed), s["positions"], s["masses"], kT)
  st = integrator.run(st, zero, steps, dt, kT, gamma)
  return s, st


def main():
  with open(os.path.join(HERE, "known_answers.json"), "w") as f:
    json.dump(KNOWN_ANSWERS, f, indent=1)
  out = {}
  for c in CASES:
    name = c[0]
    s, cutoff = case_system(name)
    e, frc, ex = energy.energy_forces(s, s["positions"], cutoff)
    out[f"{name}/terms"] = np.array([e[t] for t in energy.TERMS + ("total",)])
    out[f"{name}/forces"] = frc
    out[f"{name}/born_radii"] = ex["born_radii"]
    out[f"{name}/positions_digest"] = np.array(positions_digest(s["positions"]))
  s, st = zero_force_run()
  name = ZERO_FORCE[0]
  out[f"{name}/position"] = st.position
  out[f"{name}/momentum"] = st.momentum
  out[f"{name}/key"] = st.key
  out[f"{name}/positions_digest"] = np.array(positions_digest(s["positions"]))
  out["term_names"] = np.array(energy.TERMS + ("total",))
  np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **out)


if __name__ == "__main__":
  main()
