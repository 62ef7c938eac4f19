"""Replica exchange (parallel tempering) on one device batch: prolix
``pt/replica_exchange.py`` and ``pt/temperature.py``.

All replicas of the system run as systems of one ragged batch, each with its
own temperature and threefry key, so one launch per kernel advances every
replica.  Every ``exchange_interval_ps`` the neighbour pairs of one phase
((0,1), (2,3), ... or (1,2), (3,4), ..., chosen with probability 1/2) swap
configurations with the Metropolis probability min(1, exp((beta_i -
beta_j)(E_i - E_j))) (replica_exchange.py:100-245): positions, momenta and
forces move between slots on the device (``pb2_permute_systems``), the
temperatures, keys and step counters stay.

Units: the reference integrates in ps with masses divided by 418.4
(replica_exchange.py:306-309, :334); this engine uses AKMA time with masses
in amu, the same dynamics.  The exchange draws come from a NumPy generator
seeded by ``key`` (not bit-identical to jax.random).
"""

from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from . import engine

BOLTZMANN_KCAL = engine.KB_KCAL


@dataclasses.dataclass
class ReplicaExchangeSpec:
  """prolix pt/replica_exchange.py:43-61."""
  n_replicas: int
  min_temp: float = 300.0
  max_temp: float = 400.0
  total_time_ns: float = 10.0
  step_size_fs: float = 2.0
  exchange_interval_ps: float = 10.0
  save_interval_ns: float = 0.01
  gamma: float = 1.0
  use_pbc: bool = False
  box: object = None
  save_path: str = "remd_trajectory.array_record"


@dataclasses.dataclass
class ReplicaExchangeState:
  """prolix pt/replica_exchange.py:64-99 (host arrays).  positions[i] is the
  configuration at temperatures[i]; walker_indices[i] the walker holding it."""
  positions: np.ndarray
  velocities: np.ndarray
  forces: np.ndarray
  mass: np.ndarray
  walker_indices: np.ndarray
  step: int
  time_ns: float
  potential_energy: np.ndarray
  kinetic_energy: np.ndarray
  exchange_attempts: int = 0
  exchange_successes: int = 0

  def replace(self, **kwargs):
    return dataclasses.replace(self, **kwargs)


def generate_temperature_ladder(n_replicas: int, min_temp: float, max_temp: float,
                                geometric: bool = True) -> np.ndarray:
  """prolix pt/temperature.py:13-45."""
  if n_replicas < 1:
    raise ValueError("n_replicas must be >= 1")
  if n_replicas == 1:
    return np.array([float(min_temp)])
  if geometric:
    return np.exp(np.linspace(math.log(min_temp), math.log(max_temp), n_replicas))
  return np.linspace(min_temp, max_temp, n_replicas)


def exchange_permutation(energies, temperatures, rng):
  """One exchange attempt (replica_exchange.py:100-245).  Returns
  (perm, attempts, accepted): slot i takes the configuration of slot
  perm[i]."""
  e = np.asarray(energies, np.float64)
  betas = 1.0 / (BOLTZMANN_KCAL * np.asarray(temperatures, np.float64))
  n = e.shape[0]
  offset = 1 if rng.random() < 0.5 else 0
  i = np.arange(offset, n - 1, 2)
  j = i + 1
  delta = (betas[i] - betas[j]) * (e[i] - e[j])
  prob = np.exp(np.minimum(0.0, delta))
  accept = rng.random(i.shape[0]) < prob
  perm = np.arange(n)
  perm[i] = np.where(accept, j, i)
  perm[j] = np.where(accept, i, j)
  return perm, int(i.shape[0]), int(np.sum(accept))


def run_replica_exchange(system_params, r_init, spec: ReplicaExchangeSpec, key=None, device: int = 0,
                         n_intervals: int | None = None) -> ReplicaExchangeState:
  """prolix pt/replica_exchange.py:248-459 on one device batch.

  ``r_init``: (N, 3) or (n_replicas, N, 3).  ``n_intervals`` overrides the
  number of exchange intervals derived from ``total_time_ns``.
  """
  if spec.use_pbc:
    raise NotImplementedError("prolix_b200 implements the implicit-solvent path only")
  from .system import system_to_dict
  sysd = system_to_dict(system_params)
  n_rep = int(spec.n_replicas)
  temps = generate_temperature_ladder(n_rep, spec.min_temp, spec.max_temp)
  r = np.asarray(r_init, np.float64)
  r = np.broadcast_to(r, (n_rep,) + r.shape[-2:]) if r.ndim == 2 else r
  if key is None:
    key = (0, int(time.time()) & 0xFFFFFFFF)
  k0, k1 = (int(v) & 0xFFFFFFFF for v in np.asarray(key).reshape(2))
  rng = np.random.default_rng([k0, k1])
  origin = engine.default_origin(r[0])
  dt = engine.akma_dt(spec.step_size_fs)
  replicas = [dict(sysd, positions=r[i], kT=BOLTZMANN_KCAL * float(temps[i]), dt=dt,
                   gamma=engine.akma_gamma(spec.gamma), key=(k0, (k1 + 7919 * (i + 1)) & 0xFFFFFFFF),
                   origin=origin) for i in range(n_rep)]
  steps_per_exchange = max(1, round(spec.exchange_interval_ps / (spec.step_size_fs * 1e-3)))
  total = n_intervals if n_intervals is not None else int(spec.total_time_ns * 1000 / spec.exchange_interval_ps)
  walker = np.arange(n_rep)
  attempts = successes = 0
  masses = np.asarray(sysd["masses"], np.float64)
  with engine.Batch(replicas, device=device) as b:
    b.langevin_init()
    energies = b.energy_forces()[0][:, -1]
    for _ in range(total):
      b.langevin_run(steps_per_exchange)
      energies = b.energy_forces()[0][:, -1]
      perm, a, s = exchange_permutation(energies, temps, rng)
      attempts += a
      successes += s
      if np.any(perm != np.arange(n_rep)):
        b.permute_systems(perm)
        walker = walker[perm]
        energies = energies[perm]
    st = b.get_state(fields=("position", "momentum", "force", "step"))
  n = masses.shape[0]
  p = st["momentum"].reshape(n_rep, n, 3)
  ke = 0.5 * np.sum(p ** 2 / masses[None, :, None], axis=(1, 2))
  return ReplicaExchangeState(
      positions=st["position"].reshape(n_rep, n, 3), velocities=p / masses[None, :, None],
      forces=st["force"].reshape(n_rep, n, 3), mass=masses, walker_indices=walker,
      step=int(st["step"][0]), time_ns=float(st["step"][0] * spec.step_size_fs * 1e-6),
      potential_energy=np.asarray(energies), kinetic_energy=ke,
      exchange_attempts=attempts, exchange_successes=successes)
