"""Pins the CPU oracle against the known answers the reference's own tests
hold for this path, and against published known-answer vectors of the
third-party algorithms on the path.  CPU only."""

import json
import math
import os

import numpy as np
import pytest

from oracle import bonded, energy, gbsa, integrator, prng
from prolix_b200 import synth

TAU = 1.0 / 1.0 - 1.0 / 78.5
with open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")) as _f:
  KA = json.load(_f)


def gb_only(system, pos, cutoff=0.0):
  s = dict(system)
  s["sigmas"] = np.ones(len(pos))
  s["epsilons"] = np.zeros(len(pos))
  e, f, ex = gbsa.nonbonded(s, pos, cutoff, k_coul=0.0, ace=False)
  return e["gb"], f, ex


def test_born_ion():
  # prolix tests/physics/test_generalized_born.py:11-52: a single ion of
  # radius 2.0 has Born radius 2.0 - 0.09 and E = -1/2 k tau q^2 / B.
  ka = KA["born_ion"]
  s = {"charges": [ka["charge"]], "radii": [ka["radius"]], "scaled_radii": [ka["radius"]]}
  e, _, ex = gb_only(s, np.zeros((1, 3)))
  assert ex["born_radii"][0] == pytest.approx(ka["born_radius"], rel=1e-12)
  assert e == pytest.approx(ka["gb_energy"], rel=ka["gb_energy_rel"])


def test_gb_gradient_matches_finite_difference():
  # prolix tests/physics/test_generalized_born.py:54-91 (2 atoms at 3.5 A).
  pos = np.array([[0.0, 0.0, 0.0], [3.5, 0.0, 0.0]])
  s = {"charges": [1.0, -1.0], "radii": [1.5, 1.5], "scaled_radii": [1.5, 1.5]}
  _, f, _ = gb_only(s, pos)
  h = 1e-5
  num = np.zeros_like(pos)
  for i in range(2):
    for k in range(3):
      p = pos.copy(); p[i, k] += h
      ep = gb_only(s, p)[0]
      p[i, k] -= 2 * h
      em = gb_only(s, p)[0]
      num[i, k] = -(ep - em) / (2 * h)
  np.testing.assert_allclose(f, num, rtol=1e-6, atol=1e-8)


def test_complete_neighbour_list_equals_dense():
  # prolix tests/physics/test_generalized_born.py:93-136: with every pair in
  # the list, the neighbour-list GB energy equals the dense one.
  pos = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0], [5.0, 0.0, 0.0]])
  s = {"charges": [0.5, -0.5, 0.5], "radii": [1.5] * 3, "scaled_radii": [1.5] * 3}
  e_dense = gb_only(s, pos)[0]
  e_nl = gb_only(s, pos, cutoff=100.0)[0]
  assert e_nl == pytest.approx(e_dense, rel=1e-12)


def test_gb_nve_drift():
  # prolix tests/physics/test_generalized_born.py:138-end: 100 velocity
  # Verlet steps of three GB particles (mass 10, dt 1e-3) drift < 1e-4.
  pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0], [0.0, 4.0, 0.0]])
  s = {"charges": [0.5, -0.5, 0.5], "radii": [1.5] * 3, "scaled_radii": [1.5] * 3}
  m = np.array([10.0, 10.0, 10.0])[:, None]
  dt = 1e-3
  v = prng.normal_f32(prng.prng_key(0), 9).astype(np.float64).reshape(3, 3) * 0.1
  e0, f, _ = gb_only(s, pos)
  e_init = e0 + 0.5 * np.sum(m * v * v)
  r = pos.copy()
  for _ in range(100):
    vh = v + 0.5 * (f / m) * dt
    r = r + vh * dt
    e, f, _ = gb_only(s, r)
    v = vh + 0.5 * (f / m) * dt
  e_fin = e + 0.5 * np.sum(m * v * v)
  assert abs(e_fin - e_init) / abs(e_init) < 1e-4


def test_bond_and_angle_known_values():
  # prolix tests/physics/test_bonded.py:10-59
  kb, ka = KA["bond"], KA["angle"]
  e, f = bonded.bonds(np.array(kb["positions"]), [[0, 1]], [kb["params"]])
  assert e == pytest.approx(kb["energy"])
  assert f[0, 0] == pytest.approx(kb["force_x"][0], abs=kb["force_abs"])
  assert f[1, 0] == pytest.approx(kb["force_x"][1], abs=kb["force_abs"])
  e, _ = bonded.angles(np.array(ka["positions"]), [[0, 1, 2]], [ka["params"]])
  assert e == pytest.approx(ka["energy"], rel=ka["energy_rel"])


def test_threefry_known_answer_vectors():
  # Random123 known-answer vectors for threefry2x32, 20 rounds
  u = np.uint32
  for key, ctr, want in KA["threefry2x32_20"]["cases"]:
    got = prng.threefry2x32(u(key[0]), u(key[1]), u(ctr[0]), u(ctr[1]))
    assert [int(got[0]), int(got[1])] == want


def test_jax_split_documented_values():
  # jax.random.split(jax.random.PRNGKey(0)) as printed in JAX's documentation,
  # for the original and the partitionable (default) key layouts.
  k = prng.prng_key(0)
  kv = KA["jax_split_prngkey0"]
  np.testing.assert_array_equal(prng.split(k, partitionable=False), kv["original"])
  np.testing.assert_array_equal(prng.split(k, partitionable=True), kv["partitionable"])


def test_normal_sampler_statistics():
  z = prng.normal_f32(prng.prng_key(11), 400_000).astype(np.float64)
  assert abs(z.mean()) < 0.01
  assert abs(z.std() - 1.0) < 0.01
  assert abs(np.mean(z ** 4) - 3.0) < 0.05
  assert z.dtype == np.float64 and np.isfinite(z).all()


def test_log1p_and_erfinv_accuracy():
  from scipy.special import erfinv
  x = np.random.default_rng(0).uniform(-0.999, 0.0, size=200_000).astype(np.float32)
  got = prng.log1p_f32(x).astype(np.float64)
  ref = np.log1p(x.astype(np.float64))
  assert np.max(np.abs(got - ref) / np.abs(ref)) < 5e-7
  u = prng.uniform_pm1(prng.random_bits32(prng.prng_key(3), 200_000))
  assert u.min() >= np.nextafter(np.float32(-1), np.float32(0)) and u.max() < 1.0
  e = prng.erfinv_f32(u).astype(np.float64)
  r = erfinv(u.astype(np.float64))
  big = np.abs(r) > 1e-3
  assert np.max(np.abs(e - r)[big] / np.abs(r[big])) < 2e-5


@pytest.mark.parametrize("cutoff", [0.0, 7.0])
def test_oracle_forces_match_finite_difference(cutoff):
  s = synth.make_chain(22, 5, compact=True, cmap=True)
  s["cmap_torsions"] = np.array([[2, 3, 4, 5, 6], [9, 10, 11, 12, 13]], dtype=np.int32)
  s["cmap_indices"] = np.array([0, 0], dtype=np.int32)
  pos = s["positions"] + np.random.default_rng(1).normal(0, 0.03, size=s["positions"].shape)
  e, f, _ = energy.energy_forces(s, pos, cutoff)
  assert all(abs(e[t]) > 0 for t in ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb"))
  h = 1e-5
  num = np.zeros_like(pos)
  for i in range(pos.shape[0]):
    for k in range(3):
      p = pos.copy(); p[i, k] += h
      ep = energy.total_energy(s, p, cutoff)
      p[i, k] -= 2 * h
      em = energy.total_energy(s, p, cutoff)
      num[i, k] = -(ep - em) / (2 * h)
  assert np.max(np.abs(num - f)) < 1e-5 * max(1.0, np.max(np.abs(f)))


def test_cmap_patch_reproduces_grid():
  g = np.random.default_rng(4).uniform(-2, 2, size=(24, 24))
  c = bonded.cmap_coefficients(g)
  # value at the patch origin is the grid value (grid stored (psi, phi))
  for i, j in [(0, 0), (5, 17), (23, 23)]:
    assert c[i, j, 0] == pytest.approx(g[j, i], abs=1e-12)
  # continuity across a patch edge in phi
  i, j = 7, 11
  u1 = np.array([1.0, 1.0, 1.0, 1.0])
  v = 0.37
  vp = np.array([1, v, v * v, v ** 3])
  left = u1 @ c[i, j].reshape(4, 4) @ vp
  right = np.array([1.0, 0, 0, 0]) @ c[i + 1, j].reshape(4, 4) @ vp
  assert left == pytest.approx(right, abs=1e-10)


def test_integrator_step_order():
  # With zero force the BAOAB update reduces to the O step plus drift.
  key = prng.prng_key(7)
  x = np.zeros((4, 3))
  st = integrator.init(lambda r: np.zeros_like(r), key, x, np.full(4, 12.0), 0.6)
  st2 = integrator.step(st, lambda r: np.zeros_like(r), 0.02, 0.6, 0.05)
  c1 = math.exp(-0.05 * 0.02)
  k2 = prng.split(st.key)
  xi = prng.normal_f32(k2[1], 12).astype(np.float64).reshape(4, 3)
  p = c1 * st.momentum + math.sqrt(1 - c1 * c1) * np.sqrt(12.0 * 0.6) * xi
  np.testing.assert_allclose(st2.momentum, p, rtol=1e-15, atol=1e-15)
  np.testing.assert_array_equal(st2.key, k2[0])
