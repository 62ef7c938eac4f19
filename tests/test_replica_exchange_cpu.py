"""Replica-exchange host logic (prolix pt/replica_exchange.py:100-245,
pt/temperature.py:13-45): temperature ladder, neighbour pairing by phase and
the Metropolis acceptance rate."""

import math

import numpy as np

from prolix_b200 import replica_exchange as rx


def test_temperature_ladder():
  t = rx.generate_temperature_ladder(4, 300.0, 400.0)
  np.testing.assert_allclose(t, 300.0 * (400.0 / 300.0) ** (np.arange(4) / 3.0))
  np.testing.assert_allclose(rx.generate_temperature_ladder(3, 300.0, 400.0, geometric=False),
                             [300.0, 350.0, 400.0])
  assert rx.generate_temperature_ladder(1, 310.0, 400.0).tolist() == [310.0]


def test_equal_temperatures_always_swap_one_phase():
  rng = np.random.default_rng(1)
  for _ in range(20):
    perm, attempts, ok = rx.exchange_permutation(np.array([1.0, 5.0, -3.0, 2.0, 0.0]),
                                                 np.full(5, 300.0), rng)
    assert ok == attempts and attempts == 2
    assert sorted(perm.tolist()) == list(range(5))
    moved = np.nonzero(perm != np.arange(5))[0]
    assert moved.tolist() in ([0, 1, 2, 3], [1, 2, 3, 4])
    assert np.all(np.abs(perm - np.arange(5)) <= 1)


def test_metropolis_rate():
  # two replicas: delta = (b0 - b1)(E0 - E1) < 0 here, so p = exp(delta)
  temps = np.array([300.0, 360.0])
  e = np.array([-100.0, -98.5])
  betas = 1.0 / (rx.BOLTZMANN_KCAL * temps)
  p = math.exp((betas[0] - betas[1]) * (e[0] - e[1]))
  assert 0.05 < p < 0.95
  rng = np.random.default_rng(7)
  acc = att = 0
  for _ in range(20000):
    _, a, s = rx.exchange_permutation(e, temps, rng)
    att += a
    acc += s
  # the odd phase has no pair for two replicas: about half the attempts are empty
  assert abs(att - 10000) < 400
  rate = acc / att
  assert abs(rate - p) < 4 * math.sqrt(p * (1 - p) / att)
