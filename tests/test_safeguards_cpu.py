"""The safeguarded step of prolix's batched Langevin integrator
(batched_simulate.py:218-382) as restated by the oracle: with every limit
off it is the plain BAOAB step bit for bit, and each limit rescales exactly
what the reference rescales and counts the step once (typing.py:559-563)."""

import math

import numpy as np

from oracle import integrator, prng


def _state(p, f=None, m=None):
  n = p.shape[0]
  m = np.full(n, 12.0) if m is None else m
  return integrator.State(np.zeros((n, 3)), p, np.zeros((n, 3)) if f is None else f, m,
                          prng.prng_key(4))


def test_all_limits_off_is_the_plain_step():
  rng = np.random.default_rng(0)
  st = integrator.State(rng.normal(size=(9, 3)), rng.normal(size=(9, 3)), rng.normal(size=(9, 3)),
                        rng.uniform(1, 16, 9), prng.prng_key(11))
  force = lambda r: np.sin(r)
  a = integrator.step(st, force, 0.02, 0.6, 0.05)
  counts = np.zeros(4, np.int64)
  b = integrator.step_guarded(st, force, 0.02, 0.6, 0.05, (0.0, 0.0, 0.0), counts)
  for name in ("position", "momentum", "force", "key"):
    np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
  assert not counts.any()


def test_speed_limit_scales_only_fast_atoms():
  # gamma = 0 and F = 0: the O step leaves p alone, so the limit is visible
  p = np.array([[120.0, 0.0, 0.0], [0.0, 6.0, 0.0]])  # |v| = 10 and 0.5 at m = 12
  counts = np.zeros(4, np.int64)
  zero = lambda r: np.zeros_like(r)
  out = integrator.step_guarded(_state(p), zero, 0.01, 0.6, 0.0, (2.0, 0.0, 0.0), counts)
  v = np.linalg.norm(out.momentum / 12.0, axis=1)
  assert math.isclose(v[0], 2.0, rel_tol=1e-15)
  np.testing.assert_array_equal(out.momentum[1], p[1])
  np.testing.assert_allclose(out.position[0], [0.01 * 2.0, 0, 0], rtol=1e-14)
  assert counts.tolist() == [1, 0, 0, 0]


def test_displacement_cap_scales_position_and_momentum():
  p = np.array([[120.0, 0.0, 0.0], [0.0, 1.2, 0.0]])  # moves 0.1 and 0.001 per unit-dt step
  counts = np.zeros(4, np.int64)
  zero = lambda r: np.zeros_like(r)
  out = integrator.step_guarded(_state(p), zero, 0.01, 0.6, 0.0, (0.0, 0.05, 0.0), counts)
  assert math.isclose(np.linalg.norm(out.position[0]), 0.05, rel_tol=1e-14)
  np.testing.assert_allclose(out.momentum[0], p[0] * 0.5, rtol=1e-14)
  np.testing.assert_array_equal(out.momentum[1], p[1])
  assert counts.tolist() == [0, 0, 0, 1]


def test_force_cap_applies_to_the_closing_force_only():
  # the opening force (the state's) is used as it is; the closing force is
  # capped, stored capped and counted
  big = np.array([[3e4, 4e4, 0.0], [1.0, 0.0, 0.0]])
  p = np.zeros((2, 3))
  counts = np.zeros(4, np.int64)
  out = integrator.step_guarded(_state(p, f=big.copy()), lambda r: big.copy(), 1e-4, 0.6, 0.0,
                                (0.0, 0.0, 1e4), counts)
  assert math.isclose(np.linalg.norm(out.force[0]), 1e4, rel_tol=1e-14)
  np.testing.assert_array_equal(out.force[1], big[1])
  # p = dt/2 * big (opening, uncapped) + dt/2 * capped (closing)
  np.testing.assert_allclose(out.momentum[0], 0.5e-4 * big[0] + 0.5e-4 * big[0] * 0.2, rtol=1e-14)
  assert counts.tolist() == [0, 1, 0, 0]
  # the next step opens with the stored (capped) force
  out2 = integrator.step_guarded(out, lambda r: np.zeros_like(r), 1e-4, 0.6, 0.0, (0.0, 0.0, 1e4), counts)
  np.testing.assert_allclose(out2.momentum[0], out.momentum[0] + 0.5e-4 * out.force[0], rtol=1e-14)
  assert counts.tolist() == [0, 1, 0, 0]
