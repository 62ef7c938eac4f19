"""Minimiser restatement (oracle/minimize.py) on toy force fields: FIRE's
time-step and mixing rules, the displacement cap, the lowest-RMS snapshot,
and restrained steepest descent."""

import numpy as np

from oracle import minimize as om


def test_fire_converges_on_a_harmonic_well():
  rng = np.random.default_rng(0)
  r_start = rng.normal(size=(10, 3))
  kspring = rng.uniform(1.0, 5.0, size=(10, 1))
  force_fn = lambda r: -kspring * r
  masses = np.full(10, 12.0)
  best, final = om.fire(None, r_start, r_start, np.zeros(10), masses, 400, 0.0, 0.01, 0.1, 0.1,
                        force_fn=force_fn)
  rms0 = np.sqrt(np.mean(np.sum((kspring * r_start) ** 2, axis=1)))
  rms = np.sqrt(np.mean(np.sum((kspring * best) ** 2, axis=1)))
  assert rms < 1e-3 * rms0


def test_fire_step_is_capped_and_best_snapshot_kept():
  # a steep constant force: every step hits the 0.05 A cap
  force_fn = lambda r: np.full_like(r, 1e4)
  r0 = np.zeros((4, 3))
  best, final = om.fire(None, r0, r0, np.zeros(4), np.ones(4), 3, 0.0, 0.01, 0.1, 0.05,
                        force_fn=force_fn)
  step = np.linalg.norm(final - r0, axis=1)
  assert np.all(step <= 3 * 0.05 + 1e-12)
  assert np.array_equal(best, r0)  # the constant force never lowers the RMS


def test_restrained_descent_returns_to_reference():
  r0 = np.zeros((5, 3))
  start = np.full((5, 3), 0.3)
  sel = np.array([1, 1, 0, 1, 0], dtype=float)
  r = om.steepest_descent(None, start, r0, sel, 200, 100.0, 0.002, 0.01,
                          force_fn=lambda x: np.zeros_like(x))
  # steepest descent moves from `start` toward r0 only where the restraint acts
  np.testing.assert_allclose(r[sel == 0], start[sel == 0])
  assert np.all(np.abs(r[sel == 1]) < 1e-3)


def test_restraint_and_nan_guard():
  r0 = np.zeros((3, 3))
  r = np.ones((3, 3))
  f = om.total_force(None, r, r0, 50.0, np.array([1.0, 0.0, 1.0]),
                     force_fn=lambda x: np.array([[np.nan, 1.0, 2.0], [0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]))
  np.testing.assert_array_equal(f, [[0.0, -49.0, -48.0], [0.0, 0.0, 0.0], [-49.0, -49.0, -49.0]])


def test_lbfgs_restatement_minimises_a_quadratic():
  rng = np.random.default_rng(3)
  a = rng.normal(size=(12, 12))
  hmat = a @ a.T + 12 * np.eye(12)
  x_star = rng.normal(size=(4, 3))

  def energy_fn(r):
    d = (r - x_star).reshape(-1)
    return 0.5 * d @ hmat @ d, -(hmat @ d).reshape(4, 3)

  x = om.lbfgs(None, np.zeros((4, 3)), 200, tol=1e-9, max_step=1.0, energy_fn=energy_fn)
  assert np.max(np.abs(x - x_star)) < 1e-6
