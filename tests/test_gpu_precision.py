"""Precision study (the 20,000-atom globule and the 2,500-atom 20 A case):
per-term energies and forces of the FP32/fixed-point GPU path against the
FP64 oracle (C/OpenMP restatement for the pair terms, NumPy for CMAP), and
the NVE energy drift with FP64 integrator state.

Tolerances: force relative RMS <= 1e-5; per-term energy relative <= 1e-6
(absolute floor 1e-6 kcal/mol)."""

import numpy as np
import pytest

from oracle import bonded as obonded
from oracle import cforces, prng
from prolix_b200 import engine, synth
from prolix_b200._lib import TERM_NAMES
from prolix_b200.simulate import run_minimization
from prolix_b200.system import exclusion_spec_from_bonds, make_energy_fn

pytestmark = pytest.mark.gpu


def oracle(s, cutoff, gb_cutoff):
  e, f = cforces.energy_forces(s, cutoff=cutoff, gb_cutoff=gb_cutoff)
  ec, fc = obonded.cmap(np.asarray(s["positions"]), s["cmap_torsions"], s["cmap_indices"],
                        s["cmap_energy_grids"])
  e = dict(e)
  e["cmap"] = ec
  e["total"] += ec
  for k in ("improper", "urey_bradley", "exception"):  # none in these systems
    e.setdefault(k, 0.0)
  return e, f + fc


def report(tag, e_gpu, f_gpu, e_ref, f_ref):
  rr = float(np.linalg.norm(f_gpu - f_ref) / np.linalg.norm(f_ref))
  rel = {k: abs(e_gpu[i] - e_ref[k]) / max(abs(e_ref[k]), 1e-30)
         for i, k in enumerate(TERM_NAMES) if k != "total"}
  print(f"{tag}: force rel RMS {rr:.2e}; energy rel " +
        " ".join(f"{k}={v:.1e}" for k, v in rel.items()))
  return rr


@pytest.fixture(scope="module")
def globule20k():
  return synth.make_chain(20000, 4242, compact=True, cmap=True)


@pytest.mark.parametrize("cutoff", [0.0, 20.0])
def test_globule_20k_terms_and_forces(globule20k, cutoff):
  s = globule20k
  with engine.Batch([s], cutoff=cutoff) as b:
    e, f = b.energy_forces()
  e_ref, f_ref = oracle(s, cutoff, None)
  rr = report(f"N=20000 cutoff={cutoff}", e[0], f, e_ref, f_ref)
  assert rr < 1e-5
  for i, k in enumerate(TERM_NAMES):
    if k != "total":
      assert abs(e[0][i] - e_ref[k]) <= 1e-6 * abs(e_ref[k]) + 1e-6, k


def test_config2_n2500_cutoff20_with_cmap():
  s = synth.make_chain(2500, 2500, compact=True, cmap=True)
  with engine.Batch([s], cutoff=20.0, skin=2.0) as b:
    e, f = b.energy_forces()
    b.nl_build()
  e_ref, f_ref = oracle(s, 20.0, None)
  assert report("N=2500 cutoff=20", e[0], f, e_ref, f_ref) < 1e-5
  for i, k in enumerate(TERM_NAMES):
    if k != "total":
      assert abs(e[0][i] - e_ref[k]) <= 1e-6 * abs(e_ref[k]) + 1e-6, k


def test_nve_drift_20k():
  # With the generator's default ranges (|q| <= 0.8 e on sites with sigma down
  # to 1 A) opposite charges meet in ~0.55 A wells whose compressed LJ wall
  # is stiffer than 1e5 kcal/mol/A^2, so omega * dt > 2 for hydrogen masses
  # even at 0.5 fs and no integrator holds the energy; the drift is measured
  # on the same 20,000-atom globule with physical cores (|q| <= 0.5 e, sigma
  # 2.4-3.4 A, epsilon 0.03-0.2).  The generated chain is also far from
  # equilibrium, so the run follows prolix's protocol: steepest descent,
  # Langevin thermalisation (2 ps at 1 fs, gamma 5/ps), then 1,000 velocity
  # Verlet steps (gamma = 0) at dt = 0.5 fs with FP64 integrator state.  H is
  # sampled every 100 steps; drift = |mean of the last 3 samples - mean of
  # the first 3| / |mean H|.
  s = synth.make_chain(20000, 4242, compact=True, cmap=True, **synth.PHYSICAL_RANGES)
  m = np.asarray(s["masses"])[:, None]
  efn = make_energy_fn(None, s, implicit_solvent=True, cutoff=0.0,
                       exclusion_spec=exclusion_spec_from_bonds(s["bonds"], len(s["charges"])))
  r = run_minimization(efn, s["positions"], sd_steps=100)
  efn.close()
  s_min = dict(s, positions=r)
  with engine.Batch([s_min], key=prng.prng_key(19), dt=engine.akma_dt(1.0),
                    kT=300 * engine.KB_KCAL, gamma=engine.akma_gamma(5.0)) as b:
    b.langevin_init()
    b.langevin_run(2000)
    st0 = b.get_state()
  assert np.isfinite(st0["position"]).all()
  hs = []
  with engine.Batch([dict(s_min, positions=st0["position"])], key=prng.prng_key(20),
                    dt=engine.akma_dt(0.5), kT=300 * engine.KB_KCAL, gamma=0.0) as b:
    b.set_state(position=st0["position"], momentum=st0["momentum"])
    for k in range(11):
      if k:
        b.langevin_run(100)
      st = b.get_state()
      e, _ = b.energy_forces()
      hs.append(e[0][-1] + 0.5 * np.sum(st["momentum"] ** 2 / m))
  hs = np.array(hs)
  drift = abs(hs[-3:].mean() - hs[:3].mean()) / abs(hs.mean())
  print(f"N=20000 NVE 1000 steps dt=0.5 fs after SD + 2 ps Langevin: |dH|/|H| = {drift:.2e}, "
        f"H std {hs.std():.3f}, H = {hs.mean():.1f}")
  # the reference's own NVE bound (tests/physics/test_generalized_born.py:138-end)
  assert drift < 1e-4
