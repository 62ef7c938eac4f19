"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances: per-term energies relative 1e-6 (absolute floor 1e-6 kcal/mol
per term), forces relative RMS <= 1e-5 (||F_gpu - F_ref|| / ||F_ref||).
"""

import math

import numpy as np
import pytest

from oracle import energy as oenergy
from oracle import integrator as ointeg
from oracle import prng
from prolix_b200 import engine, synth
from prolix_b200._lib import TERM_NAMES, USE_ALL, USE_BONDED, USE_CMAP

pytestmark = pytest.mark.gpu

FORCE_RRMS = 1e-5
ENERGY_REL = 1e-6


def rel_rms(a, b):
  return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def check_energies(e_gpu_row, e_ref, rel=ENERGY_REL, floor=1e-6):
  for i, name in enumerate(TERM_NAMES):
    if name == "total":
      continue
    ref = e_ref[name]
    got = e_gpu_row[i]
    assert abs(got - ref) <= rel * abs(ref) + floor, (name, got, ref)


@pytest.fixture(scope="module")
def chain166():
  return synth.make_chain(166, 1, compact=False, cmap=True)


def test_energy_forces_all_pairs_n166(chain166):
  s = chain166
  with engine.Batch([s]) as b:
    e, f = b.energy_forces()
  e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"])
  check_energies(e[0], e_ref)
  assert rel_rms(f, f_ref) < FORCE_RRMS


def test_born_radii_n166(chain166):
  s = chain166
  with engine.Batch([s]) as b:
    born = b.born_radii()
  _, _, ex = oenergy.energy_forces(s, s["positions"])
  np.testing.assert_allclose(born, ex["born_radii"], rtol=2e-6)


def test_perturbed_geometry_all_terms():
  s = synth.make_chain(300, 3, compact=True, cmap=True)
  pos = s["positions"] + np.random.default_rng(2).normal(0, 0.05, size=s["positions"].shape)
  s = dict(s, positions=pos)
  with engine.Batch([s]) as b:
    e, f = b.energy_forces()
  e_ref, f_ref, _ = oenergy.energy_forces(s, pos)
  check_energies(e[0], e_ref)
  assert rel_rms(f, f_ref) < FORCE_RRMS


def test_cutoff_mode_n600():
  s = synth.make_chain(600, 4, compact=True)
  with engine.Batch([s], cutoff=9.0) as b:
    e, f = b.energy_forces()
  e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"], cutoff=9.0)
  check_energies(e[0], e_ref)
  assert rel_rms(f, f_ref) < FORCE_RRMS


def test_globule_n2500_all_pairs():
  s = synth.make_chain(2500, 9, compact=True, cmap=True)
  with engine.Batch([s]) as b:
    e, f = b.energy_forces()
  e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"])
  check_energies(e[0], e_ref)
  assert rel_rms(f, f_ref) < FORCE_RRMS


def test_ragged_batch_matches_each_system_alone():
  systems = [synth.make_chain(n, 100 + k, compact=True) for k, n in enumerate([37, 150, 513, 64, 1000])]
  with engine.Batch(systems) as b:
    e_all, f_all = b.energy_forces()
  for k, s in enumerate(systems):
    with engine.Batch([s]) as b1:
      e1, f1 = b1.energy_forces()
    lo, hi = sum(len(x["charges"]) for x in systems[:k]), sum(len(x["charges"]) for x in systems[:k + 1])
    np.testing.assert_array_equal(f_all[lo:hi], f1)
    np.testing.assert_array_equal(e_all[k], e1[0])


def test_forces_are_deterministic():
  s = synth.make_chain(700, 5, compact=True)
  with engine.Batch([s]) as b:
    f1 = b.forces()
    f2 = b.forces()
  np.testing.assert_array_equal(f1, f2)


def test_born_ion_and_single_atom():
  s = {"positions": np.zeros((1, 3)), "charges": [1.0], "sigmas": [1.0], "epsilons": [0.1],
       "radii": [2.0], "scaled_radii": [2.0], "masses": [12.0]}
  with engine.Batch([s]) as b:
    e, f = b.energy_forces()
    born = b.born_radii()
  assert born[0] == pytest.approx(1.91, rel=1e-6)
  tau = 1.0 - 1.0 / 78.5
  assert e[0][TERM_NAMES.index("gb")] == pytest.approx(-0.5 * 332.0637 * tau / 1.91, rel=1e-6)
  assert np.all(f == 0.0)


def test_langevin_zero_force_is_bit_exact():
  # With every term disabled the integrator sees F = 0, so positions and
  # momenta must equal the FP64 oracle bit for bit (noise included).
  s = synth.make_chain(97, 21, compact=True)
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  key = prng.prng_key(1234)
  with engine.Batch([s], terms=0, key=key, dt=dt, kT=kT, gamma=gamma) as b:
    b.langevin_init()
    b.langevin_run(7)
    st = b.get_state()
  zero = lambda r: np.zeros_like(r)
  o = ointeg.init(zero, key, s["positions"], s["masses"], kT)
  o = ointeg.run(o, zero, 7, dt, kT, gamma)
  np.testing.assert_array_equal(st["momentum"], o.momentum)
  np.testing.assert_array_equal(st["position"], o.position)
  np.testing.assert_array_equal(st["key"][0], o.key)
  assert st["step"][0] == 7


def test_langevin_bonded_only_tracks_oracle():
  s = synth.make_chain(120, 8, compact=True, cmap=True)
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  key = prng.prng_key(99)
  with engine.Batch([s], terms=USE_BONDED | USE_CMAP, key=key, dt=dt, kT=kT, gamma=gamma) as b:
    b.langevin_init()
    b.langevin_run(20)
    st = b.get_state()
  from oracle import bonded
  force = lambda r: bonded.bonded_all(s, r)[1]
  o = ointeg.init(force, key, s["positions"], s["masses"], kT)
  o = ointeg.run(o, force, 20, dt, kT, gamma)
  np.testing.assert_allclose(st["position"], o.position, rtol=0, atol=1e-8)
  np.testing.assert_allclose(st["momentum"], o.momentum, rtol=0, atol=1e-7)


def test_graph_chunks_equal_eager_steps():
  s = synth.make_chain(200, 31, compact=True)
  key = prng.prng_key(5)
  with engine.Batch([s], key=key, graph_chunk=4) as b:
    b.langevin_init()
    b.langevin_run(10)
    st_graph = b.get_state()
  with engine.Batch([s], key=key) as b:
    b.set_profiling(True)  # eager launches, no graphs
    b.langevin_init()
    b.langevin_run(10)
    st_eager = b.get_state()
  np.testing.assert_array_equal(st_graph["position"], st_eager["position"])
  np.testing.assert_array_equal(st_graph["momentum"], st_eager["momentum"])
  np.testing.assert_array_equal(st_graph["key"], st_eager["key"])


def test_full_langevin_short_run_stays_close_to_oracle():
  s = synth.make_chain(166, 1, compact=False)
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  key = prng.prng_key(3)
  with engine.Batch([s], key=key, dt=dt, kT=kT, gamma=gamma) as b:
    b.langevin_init()
    b.langevin_run(10)
    st = b.get_state()
  force = lambda r: oenergy.energy_forces(s, r)[1]
  o = ointeg.init(force, key, s["positions"], s["masses"], kT)
  o = ointeg.run(o, force, 10, dt, kT, gamma)
  assert np.max(np.abs(st["position"] - o.position)) < 1e-6
  assert rel_rms(st["force"], o.force) < 1e-5


def test_nve_energy_drift_all_pairs():
  s = synth.make_chain(400, 12, compact=True)
  dt = engine.akma_dt(0.5)
  with engine.Batch([s], key=prng.prng_key(8), dt=dt, kT=300 * engine.KB_KCAL, gamma=0.0) as b:
    b.langevin_init()
    st0 = b.get_state()
    e0, _ = b.energy_forces()
    m = np.asarray(s["masses"])[:, None]
    ke0 = 0.5 * np.sum(st0["momentum"] ** 2 / m)
    b.langevin_run(1000)
    st1 = b.get_state()
    e1, _ = b.energy_forces()
  ke1 = 0.5 * np.sum(st1["momentum"] ** 2 / m)
  h0 = e0[0][-1] + ke0
  h1 = e1[0][-1] + ke1
  assert abs(h1 - h0) / abs(h0) < 1e-4
