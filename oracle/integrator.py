"""BAOAB Langevin integrator in FP64 (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows prolix physics/settle.py:1676-1744 (``langevin_with_constraints``
with no constraint) and its step helpers :2064-2087, which carry the same
B-A-O-A-F-B order as jax_md's ``nvt_langevin``:

  p += dt/2 F;  x += dt/2 p/m;
  (key, split) = split(key);  xi = normal(split, (N, 3));
  p = c1 p + c2 sqrt(m kT) xi,  c1 = exp(-gamma dt), c2 = sqrt(1 - c1^2);
  x += dt/2 p/m;  F = force(x);  p += dt/2 F.

``step_guarded`` adds the speed, displacement and force limits of prolix's
batched step (batched_simulate.py:218-382).

Init (:1676-1696): (key, split) = split(key); p = sqrt(m kT) normal(split);
F = force(x).  Units are AKMA (A, kcal/mol, amu, tau = 48.88821291839 fs;
prolix simulate.py:56-57, 770-772).
"""

from __future__ import annotations

import math

import numpy as np

from . import prng

AKMA_TIME_FS = 48.88821291839
KB_KCAL = 0.0019872041


def akma_dt(dt_fs: float) -> float:
  return dt_fs / AKMA_TIME_FS


def akma_gamma(gamma_per_ps: float) -> float:
  return gamma_per_ps * AKMA_TIME_FS * 1e-3


def kT_of(temperature_k: float) -> float:
  return temperature_k * KB_KCAL


class State:
  def __init__(self, x, p, f, m, key):
    self.position = np.asarray(x, np.float64)
    self.momentum = np.asarray(p, np.float64)
    self.force = np.asarray(f, np.float64)
    self.mass = np.asarray(m, np.float64).reshape(-1, 1)
    self.key = np.asarray(key, np.uint32)


def init(force_fn, key, x, mass, kT, partitionable=True, center=False):
  key = np.asarray(key, np.uint32)
  ks = prng.split(key, 2, partitionable)
  key, sub = ks[0], ks[1]
  x = np.asarray(x, np.float64)
  m = np.asarray(mass, np.float64).reshape(-1, 1)
  xi = prng.normal_f32(sub, x.size, partitionable).astype(np.float64).reshape(x.shape)
  p = np.sqrt(m * kT) * xi
  if center and x.shape[0] > 1:
    p = p - p.mean(axis=0, keepdims=True)
  return State(x, p, force_fn(x), m, key)


def step(state, force_fn, dt, kT, gamma, partitionable=True):
  m = state.mass
  p = state.momentum + 0.5 * dt * state.force
  x = state.position + 0.5 * dt * (p / m)
  c1 = math.exp(-gamma * dt)
  c2 = math.sqrt(1.0 - c1 * c1)
  ks = prng.split(state.key, 2, partitionable)
  key, sub = ks[0], ks[1]
  xi = prng.normal_f32(sub, x.size, partitionable).astype(np.float64).reshape(x.shape)
  p = c1 * p + c2 * np.sqrt(m * kT) * xi
  x = x + 0.5 * dt * (p / m)
  f = force_fn(x)
  p = p + 0.5 * dt * f
  return State(x, p, f, m, key)


def _norm(v, eps):
  """sqrt(|v|^2 + eps) per row, summed x, y, z in that order."""
  return np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2] + eps)[:, None]


def step_guarded(state, force_fn, dt, kT, gamma, guards, counts, partitionable=True):
  """One step of prolix's batched Langevin step without constraints
  (batched_simulate.py:218-382): the step above plus its safeguards.
  guards = (vlimit, max_dx, force_cap), each <= 0 off.  counts: int array
  of 4 in warn_counts order (typing.py:559-563), incremented in place when
  a safeguard fires on any atom (:361-367).  state.force opens the step as
  it is; the closing force is capped and stored capped (:333-340)."""
  vlimit, max_dx, force_cap = guards
  m = state.mass
  p = state.momentum + 0.5 * dt * state.force
  if vlimit > 0:  # :268-274
    vm = _norm(p / m, 1e-30)
    over = vm > vlimit
    p = np.where(over, p * np.minimum(1.0, vlimit / (vm + 1e-30)), p)
    counts[0] += int(over.any())
  x_old = state.position
  x = x_old + 0.5 * dt * (p / m)
  c1 = math.exp(-gamma * dt)
  c2 = math.sqrt(1.0 - c1 * c1)
  ks = prng.split(state.key, 2, partitionable)
  key, sub = ks[0], ks[1]
  xi = prng.normal_f32(sub, x.size, partitionable).astype(np.float64).reshape(x.shape)
  p = c1 * p + c2 * np.sqrt(m * kT) * xi
  x = x + 0.5 * dt * (p / m)
  if max_dx > 0:  # :290-305
    dr = x - x_old
    dm = _norm(dr, 1e-30)
    sc = np.minimum(1.0, max_dx / dm)
    x = x_old + dr * sc
    over = dm > max_dx
    p = np.where(over, p * sc, p)
    counts[3] += int(over.any())
  f = force_fn(x)
  if force_cap > 0:  # :336-340
    fm = _norm(f, 1e-12)
    counts[1] += int((fm > force_cap).any())
    f = f * np.minimum(1.0, force_cap / fm)
  p = p + 0.5 * dt * f
  return State(x, p, f, m, key)


def run(state, force_fn, n_steps, dt, kT, gamma, partitionable=True, guards=None, counts=None):
  """n_steps steps; with ``guards`` the safeguarded step, its counts added
  to ``counts`` (a length-4 int array)."""
  for _ in range(n_steps):
    if guards is None:
      state = step(state, force_fn, dt, kT, gamma, partitionable)
    else:
      state = step_guarded(state, force_fn, dt, kT, gamma, guards, counts, partitionable)
  return state
