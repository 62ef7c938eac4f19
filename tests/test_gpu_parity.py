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


def test_langevin_zero_force_ragged_batch_is_bit_exact():
  # The plain step over a ragged batch of block-boundary sizes (one atom,
  # partial and whole 32-atom blocks) and larger systems, about 11,000
  # blocks in all: several per resident warp, each stepped while the warp
  # copies in its next one, which often belongs to another system.  Every
  # system equals the FP64 oracle bit for bit.
  sizes = (1, 31, 32, 33, 97, 2, 64, 65) + tuple(1500 + 23 * k for k in range(120))
  keys = [prng.prng_key(500 + k) for k in range(len(sizes))]
  systems = [dict(synth.make_chain(n, 600 + n, compact=True), key=k) for n, k in zip(sizes, keys)]
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  with engine.Batch(systems, terms=0, dt=dt, kT=kT, gamma=gamma) as b:
    b.langevin_init()
    b.langevin_run(5)
    st = b.get_state()
  zero = lambda r: np.zeros_like(r)
  for k, s in enumerate(systems):
    lo, hi = b.offsets[k], b.offsets[k + 1]
    o = ointeg.init(zero, keys[k], s["positions"], s["masses"], kT)
    o = ointeg.run(o, zero, 5, dt, kT, gamma)
    np.testing.assert_array_equal(st["momentum"][lo:hi], o.momentum)
    np.testing.assert_array_equal(st["position"][lo:hi], o.position)
    np.testing.assert_array_equal(st["key"][k], o.key)


def test_new_langevin_parameters_mid_run_are_bit_exact():
  # F = 0: 3 steps, then new dt, kT and gamma for 4 more, equal the oracle's
  # steps with those arguments bit for bit (noise and its amplitude)
  s = synth.make_chain(83, 19, compact=True)
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  dt2, kT2, gamma2 = engine.akma_dt(0.5), 450 * engine.KB_KCAL, engine.akma_gamma(5.0)
  key = prng.prng_key(808)
  with engine.Batch([s], terms=0, key=key, dt=dt, kT=kT, gamma=gamma) as b:
    b.langevin_init()
    b.langevin_run(3)
    b.set_langevin_params(dt=dt2, kT=kT2, gamma=gamma2)
    b.langevin_run(4)
    st = b.get_state()
  zero = lambda r: np.zeros_like(r)
  o = ointeg.init(zero, key, s["positions"], s["masses"], kT)
  o = ointeg.run(o, zero, 3, dt, kT, gamma)
  o = ointeg.run(o, zero, 4, dt2, kT2, gamma2)
  np.testing.assert_array_equal(st["momentum"], o.momentum)
  np.testing.assert_array_equal(st["position"], o.position)


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


def test_nve_three_gb_particles():
  # prolix tests/physics/test_generalized_born.py:138-end restated: three GB
  # particles (mass 10, radius 1.5), 100 velocity Verlet steps of dt = 1e-3,
  # initial velocities 0.1 * normal(key 0); |dH| / |H| < 1e-4.
  s = {"positions": np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [0.0, 4.0, 0.0]]),
       "charges": [0.5, -0.5, 0.5], "sigmas": [1.0] * 3, "epsilons": [0.0] * 3,
       "radii": [1.5] * 3, "scaled_radii": [1.5] * 3, "masses": [10.0] * 3}
  from prolix_b200._lib import USE_GB
  v = prng.normal_f32(prng.prng_key(0), 9).astype(np.float64).reshape(3, 3) * 0.1
  with engine.Batch([s], terms=USE_GB, dt=1e-3, kT=0.0, gamma=0.0) as b:
    b.set_state(momentum=10.0 * v)
    e0, _ = b.energy_forces()
    b.langevin_run(100)
    st = b.get_state()
    e1, _ = b.energy_forces()
  h0 = e0[0][-1] + 0.5 * np.sum(10.0 * v * v)
  h1 = e1[0][-1] + 0.5 * np.sum(st["momentum"] ** 2 / 10.0)
  assert abs(h1 - h0) / abs(h0) < 1e-4


def _nve_h_change(s, dt_fs, total_fs=250.0, samples=41):
  m = np.asarray(s["masses"])[:, None]
  n = int(round(total_fs / dt_fs))
  every = n // (samples - 1)
  hs = []
  with engine.Batch([s], key=prng.prng_key(8), dt=engine.akma_dt(dt_fs),
                    kT=300 * engine.KB_KCAL, gamma=0.0) as b:
    b.langevin_init()
    for k in range(samples):
      if k:
        b.langevin_run(every)
      st = b.get_state()
      e, _ = b.energy_forces()
      hs.append(e[0][-1] + 0.5 * np.sum(st["momentum"] ** 2 / m))
  hs = np.array(hs)
  return abs(hs[-8:].mean() - hs[:8].mean()), hs


def test_nve_drift_is_second_order_in_dt():
  # gamma = 0 turns BAOAB into velocity Verlet.  If the FP32 forces are the
  # gradient of the FP64 energy, the change of H over a fixed time is
  # Verlet's O(dt^2) error: halving dt divides it by ~4.  A force/energy
  # mismatch would leave a dt-independent drift.
  s = synth.make_chain(400, 12, compact=True)
  d1, h1 = _nve_h_change(s, 0.5)
  d2, h2 = _nve_h_change(s, 0.25)
  rel = d1 / abs(h1.mean())
  print(f"NVE |dH|/|H| over 250 fs: dt 0.5 fs {rel:.2e}, dt 0.25 fs {d2 / abs(h2.mean()):.2e}")
  assert rel < 2e-4
  assert d2 < 0.4 * d1


@pytest.mark.parametrize("keep_order", [False, True])
def test_checkpoint_resume_is_bit_exact(keep_order):
  # A slot's state (FP64 x, p, threefry key), its float32 frame origin and
  # its atom order fully determine the trajectory: snapshot at step 10,
  # restore into a new batch, continue -> identical to the uninterrupted run.
  # The stored atom order follows the positions a batch is created from, so
  # the new batch is created from the same description (or keeps the input
  # order, when any positions will do).
  s = synth.make_chain(420, 33, compact=True)
  s = dict(s, origin=engine.default_origin(s["positions"]))
  key = prng.prng_key(77)
  with engine.Batch([s], key=key, keep_atom_order=keep_order) as b:
    b.langevin_init()
    b.langevin_run(10)
    snap = b.get_state()
    b.langevin_run(10)
    ref = b.get_state()
  s2 = dict(s, positions=snap["position"]) if keep_order else s
  with engine.Batch([s2], key=key, keep_atom_order=keep_order) as b2:
    b2.set_state(position=snap["position"], momentum=snap["momentum"], key=snap["key"])
    b2.langevin_run(10)
    out = b2.get_state()
  np.testing.assert_array_equal(out["position"], ref["position"])
  np.testing.assert_array_equal(out["momentum"], ref["momentum"])
  np.testing.assert_array_equal(out["key"], ref["key"])


def test_full_state_restore_is_bit_exact_without_force_evaluation():
  # x, p, F and keys round-trip through page-locked host buffers; the restored
  # batch continues exactly as the uninterrupted one.
  import torch
  s = synth.make_chain(700, 34, compact=True)
  s = dict(s, origin=engine.default_origin(s["positions"]))
  key = prng.prng_key(78)
  with engine.Batch([s], key=key) as b:
    b.langevin_init()
    b.langevin_run(7)
    n = b.n_atoms
    pinned = {name: torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
              for name in ("position", "momentum", "force")}
    snap = b.get_state(fields=("position", "momentum", "force", "key"), out=pinned)
    assert snap["position"] is pinned["position"]
    snap = {k: v.copy() for k, v in snap.items()}
    b.langevin_run(9)
    ref = b.get_state()
  with engine.Batch([s], key=(1, 2)) as b2:  # same description: same stored atom order
    b2.set_full_state(snap["position"], snap["momentum"], snap["force"], key=snap["key"])
    got = b2.get_state(fields=("force",))
    np.testing.assert_array_equal(got["force"], snap["force"])
    b2.langevin_run(9)
    out = b2.get_state()
  for f in ("position", "momentum", "force", "key"):
    np.testing.assert_array_equal(out[f], ref[f])


def test_nl_born_dense_gb_split():
  # descreening and chain rule within 10 A, GB pair terms over all pairs
  # (generalized_born.py:706-817); against the FP64 restatement
  from oracle import bonded as obonded
  from oracle import gbsa as ogbsa
  s = synth.make_chain(600, 61, compact=True)
  with engine.Batch([s], cutoff=0.0, gb_cutoff=0.0, born_cutoff=10.0) as b:
    e, f = b.energy_forces()
    born = b.born_radii()
  en, fn, ex = ogbsa.nonbonded(s, s["positions"], 0.0, gb_cutoff=0.0, born_cutoff=10.0)
  _, fb = obonded.bonded_all(s, s["positions"])
  f_ref = fn + fb
  assert np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref) < 1e-5
  np.testing.assert_allclose(born, ex["born_radii"], rtol=2e-6)
  for k in ("gb", "nonpolar", "lj", "coulomb"):
    i = TERM_NAMES.index(k)
    assert abs(e[0][i] - en[k]) <= 1e-6 * abs(en[k]) + 1e-6, k
  with engine.Batch([s]) as b:  # dense Born radii differ: the option is an approximation
    born_dense = b.born_radii()
  assert np.max(np.abs(born - born_dense) / born_dense) > 1e-4
