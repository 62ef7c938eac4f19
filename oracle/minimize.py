"""Restrained steepest descent and FIRE, FP64, one system.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates the per-system minimisation stages of prolix ``batched_minimize``
(batched_simulate.py:682-960):

* restraint E = k/2 sum_i m_i |r_i - r0_i|^2 on a 0/1 selection m
  (``_selective_restraint_energy``, :675-679); non-finite force components
  are zeroed (:757-759, :840-842);
* steepest descent: dr = F dt with |dr| capped at max_dx per atom
  (:771-777);
* FIRE (jax_md 0.2.27 ``minimize.fire_descent``, a third-party dependency
  absent here; the published algorithm of Bitzek et al., PRL 97, 170201
  (2006) with its defaults n_min 5, f_inc 1.1, f_dec 0.5, alpha_start 0.1,
  f_alpha 0.99), one velocity-Verlet step on momenta followed by the FIRE
  mixing, then the reference's per-atom displacement cap with momenta
  scaled alike and the force kept from the uncapped position (:845-870),
  and the lowest-RMS snapshot taken at the start of each iteration
  (:843-849, :875-878).

Parity of the FIRE bookkeeping with jax_md is unpinned (no jax_md output
exists here); the restatement anchors on the reference's own call site.
"""

from __future__ import annotations

import numpy as np

from . import energy

N_MIN, F_INC, F_DEC, ALPHA_START, F_ALPHA = 5, 1.1, 0.5, 0.1, 0.99


def total_force(system, r, r0, k, sel, force_fn=None):
  f = (force_fn or (lambda x: energy.energy_forces(system, x)[1]))(r)
  if k:
    f = f - k * (r - r0) * sel[:, None]
  return np.where(np.isfinite(f), f, 0.0)


def steepest_descent(system, r_start, r0, sel, n_steps, k, dt, max_dx, force_fn=None):
  r = np.array(r_start, dtype=np.float64)
  for _ in range(n_steps):
    f = total_force(system, r, r0, k, sel, force_fn)
    d = f * dt
    dm = np.sqrt(np.sum(d * d, axis=1, keepdims=True) + 1e-30)
    r = r + d * np.minimum(1.0, max_dx / dm)
  return r


def fire(system, r_start, r0, sel, masses, n_steps, k, dt_start, dt_max, max_disp, force_fn=None,
         force_cap=0.0):
  """Returns the lowest-RMS positions of the stage and the final positions.
  max_disp / force_cap 0 disable the caps; the force cap scales each atom's
  state force for the first half kick (prolix simulate.py:613-621)."""
  m = np.asarray(masses, np.float64)[:, None]
  r = np.array(r_start, dtype=np.float64)
  p = np.zeros_like(r)
  f = total_force(system, r, r0, k, sel, force_fn)
  dt, alpha, npos = float(dt_start), ALPHA_START, 0
  best_r, best_rms = r.copy(), 1e10
  for _ in range(n_steps):
    rms = np.sqrt(np.sum(f * f) / r.shape[0])
    if rms < best_rms:
      best_r, best_rms = r.copy(), rms
    r_before = r
    fk = f
    if force_cap > 0:
      fk = f * np.minimum(1.0, force_cap / (np.linalg.norm(f, axis=1, keepdims=True) + 1e-8))
    p = p + 0.5 * dt * fk
    r = r + dt * p / m
    f = total_force(system, r, r0, k, sel, force_fn)
    p = p + 0.5 * dt * f
    fp = float(np.sum(f * p))
    fn = np.sqrt(np.sum(f * f) + 1e-6)
    pn = np.sqrt(np.sum(p * p))
    p = p + alpha * (f * pn / fn - p)
    npos = npos + 1 if fp >= 0 else 0
    if fp > 0 and npos > N_MIN:
      dt = min(dt * F_INC, dt_max)
      alpha = alpha * F_ALPHA
    if fp < 0:
      dt = dt * F_DEC
      alpha = ALPHA_START
      p = np.zeros_like(p)
    d = r - r_before
    sc = np.minimum(1.0, max_disp / np.sqrt(np.sum(d * d, axis=1, keepdims=True) + 1e-30)) if max_disp > 0 else 1.0
    r = r_before + d * sc
    p = p * sc
  return best_r, r


def lbfgs(system, r_start, n_iter, tol=1e-6, max_step=0.1, hist=10, max_trials=30, energy_fn=None):
  """L-BFGS (Nocedal & Wright alg. 7.4/7.5) as the device polish runs it:
  two-loop recursion with H0 = (s.y / y.y) I, backtracking from
  t = min(1, max_step) by 0.8 until E(t) <= E0 + 1e-4 t g.d and
  |g(t).d| <= 0.9 |g.d| (or the last trial), steepest descent when d is
  not a descent direction, pairs kept only with s.y > 1e-12, stop when
  |g| < tol.  (jaxopt's LBFGS, the reference's stage, is third-party and
  absent; this is the published algorithm with the reference's settings.)"""
  def ef(r):
    if energy_fn is not None:
      return energy_fn(r)
    e, f, _ = energy.energy_forces(system, r)
    return e["total"], f

  x = np.array(r_start, dtype=np.float64)
  e0, f = ef(x)
  g = np.where(np.isfinite(-f), -f, 0.0)
  hs, hy, rho = [], [], []
  for _ in range(n_iter):
    q = g.copy()
    alphas = []
    for s_, y_, r_ in zip(reversed(hs), reversed(hy), reversed(rho)):
      a_ = r_ * np.sum(s_ * q)
      alphas.append(a_)
      q = q - a_ * y_
    gamma = np.sum(hs[-1] * hy[-1]) / np.sum(hy[-1] * hy[-1]) if hs else 1.0
    q = q * gamma
    for s_, y_, r_, a_ in zip(hs, hy, rho, reversed(alphas)):
      b_ = r_ * np.sum(y_ * q)
      q = q + s_ * (a_ - b_)
    d = -q
    gd = np.sum(g * d)
    if not gd < 0:
      d = -g
      gd = -np.sum(g * g)
      hs, hy, rho = [], [], []
    t = min(1.0, max_step)
    for trial in range(max_trials):
      xt = x + t * d
      et, ft = ef(xt)
      gt = np.where(np.isfinite(-ft), -ft, 0.0)
      ok = np.isfinite(et) and et <= e0 + 1e-4 * t * gd and abs(np.sum(gt * d)) <= 0.9 * abs(gd)
      if ok or trial == max_trials - 1:
        break
      t *= 0.8
    s_, y_ = xt - x, gt - g
    sy = np.sum(s_ * y_)
    if sy > 1e-12:
      hs.append(s_); hy.append(y_); rho.append(1.0 / sy)
      if len(hs) > hist:
        hs.pop(0); hy.pop(0); rho.pop(0)
    x, g, e0 = xt, gt, et
    if np.sqrt(np.sum(g * g)) < tol:
      break
  return x
