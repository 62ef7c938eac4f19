"""Drop-ins for prolix's Langevin drivers on the implicit-solvent path.

* ``nvt_langevin(energy_fn, shift_fn, dt, kT, gamma, mass)`` returns
  ``(init_fn, apply_fn)`` with jax_md's protocol, the integrator that prolix
  uses (physics/simulate.py:245, physics/settle.py:1114-1117, 1637-1746):
  ``init_fn(key, R, mass=...)`` draws p = sqrt(m kT) normal(split(key)[1]),
  removes its mean as jax_md does (``center_velocity=True``) and evaluates
  the force; ``apply_fn(state)`` advances one BAOAB step.  The state
  stays on the GPU; its arrays are read back when accessed.
* ``run_minimization`` restates prolix's steepest descent with a 4-point
  backtracking line search (physics/simulate.py:141-196) on GPU energies and
  forces.
* ``run_simulation`` follows physics/simulate.py:357-508: minimise, thermalise
  with Langevin at dt = 2 fs, gamma = 1/ps, then optional production from a
  ``SimulationSpec``.

Units are AKMA inside the engine (A, kcal/mol, amu, tau = 48.88821291839 fs);
``run_simulation`` takes prolix's ps-based arguments and converts them.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from . import engine
from .system import EnergyFn, exclusion_spec_from_bonds, make_energy_fn, system_to_dict

BOLTZMANN_KCAL = 0.0019872041


@dataclasses.dataclass
class SimulationSpec:
  """prolix physics/simulate.py:26-52 (time in ps inside the properties)."""
  total_time_ns: float
  step_size_fs: float = 2.0
  ensemble: str = "nvt_langevin"
  temperature: float = 300.0
  pressure: float | None = None
  gamma: float = 1.0
  tau: float = 0.5
  chain_length: int = 5
  chain_steps: int = 1
  save_interval_ns: float = 0.001
  accumulate_steps: int = 500
  save_path: str = "trajectory.array_record"
  use_shake: bool = False

  @property
  def dt(self) -> float:
    return self.step_size_fs / 1000.0

  @property
  def steps(self) -> int:
    return int(self.total_time_ns * 1000.0 / self.dt)


class NVTLangevinState:
  """Device-resident BAOAB state; fields read back lazily (jax_md names)."""

  def __init__(self, batch: engine.Batch, mass):
    self._batch = batch
    self._mass = np.asarray(mass, dtype=np.float64).reshape(-1, 1)
    self._cache = None

  def _state(self):
    if self._cache is None:
      self._cache = self._batch.get_state()
    return self._cache

  @property
  def position(self):
    return self._state()["position"]

  positions = position

  @property
  def momentum(self):
    return self._state()["momentum"]

  @property
  def force(self):
    return self._state()["force"]

  @property
  def mass(self):
    return self._mass

  @property
  def rng(self):
    return self._state()["key"][0]

  key = rng

  @property
  def step(self) -> int:
    return int(self._state()["step"][0])

  def velocity(self):
    return self.momentum / self._mass


def _as_energy_fn(energy_or_force_fn) -> EnergyFn:
  if isinstance(energy_or_force_fn, EnergyFn):
    return energy_or_force_fn
  fn = getattr(energy_or_force_fn, "__self__", None)
  if isinstance(fn, EnergyFn):
    return fn
  raise TypeError("nvt_langevin needs the energy function returned by "
                  "prolix_b200.system.make_energy_fn (the GPU path carries the system)")


def _use(batch, dt: float, kT: float):
  """Make the batch step at (dt, kT), recomputing its constants only when
  they change (the recomputation is exact: equal to a batch created with
  the same values)."""
  if batch.langevin_now != (dt, kT):
    batch.set_langevin_params(dt=dt, kT=kT)
    batch.langevin_now = (dt, kT)


def nvt_langevin(energy_or_force_fn, shift_fn, dt: float, kT: float, gamma: float = 0.1,
                 mass=1.0, center_velocity: bool = True, **kwargs):
  """BAOAB Langevin (jax_md ``nvt_langevin`` protocol) on the GPU.

  dt and gamma are in the caller's time unit with masses in the matching
  unit (AKMA: dt in tau, gamma in 1/tau, masses in amu).  As in jax_md,
  ``center_velocity`` removes the mean initial momentum of a system of more
  than one atom; the draw itself is settle.py:1676-1696's.
  """
  efn = _as_energy_fn(energy_or_force_fn)

  def init_fn(key, R, mass=mass, **kw):
    _kT = float(kw.pop("kT", kT))
    n = efn.n_atoms
    m = np.broadcast_to(np.asarray(mass, dtype=np.float64).reshape(-1), (n,)).copy()
    sysd = dict(efn.system, positions=np.asarray(R, dtype=np.float64).reshape(n, 3), masses=m)
    # the momenta are drawn at init's kT (settle.py:1676-1691); the steps
    # run at the factory's kT unless a call passes its own
    batch = engine.Batch([sysd], cutoff=efn.cutoff, gb_cutoff=efn.gb_cutoff, born_cutoff=efn.born_cutoff,
                         key=np.asarray(key, dtype=np.uint32).reshape(2), dt=float(dt),
                         kT=_kT, gamma=float(gamma),
                         eps_in=efn.batch.prepared[0]["scal"]["eps_in"],
                         eps_out=efn.batch.prepared[0]["scal"]["eps_out"])
    batch.langevin_init()
    if center_velocity:
      batch.center_momentum()
    batch.langevin_now = (float(dt), _kT)
    _use(batch, float(dt), float(kT))
    return NVTLangevinState(batch, m)

  def apply_fn(state: NVTLangevinState, n_steps: int = 1, **kw):
    # per-call dt / kT overrides hold for that call only; later calls fall
    # back to the factory's values (physics/settle.py:1698-1700)
    _use(state._batch, float(kw.get("dt", dt)), float(kw.get("kT", kT)))
    state._batch.langevin_run(int(n_steps))
    return NVTLangevinState(state._batch, state._mass)

  return init_fn, apply_fn


def run_minimization(energy_fn: EnergyFn, initial_positions, steps: int = 500,
                     dt_start: float = 2e-3, dt_max: float = 4e-3,
                     max_displacement_per_step: float = 0.1, sd_steps: int = 200):
  """Steepest descent with backtracking (prolix physics/simulate.py:141-196)."""
  r = np.asarray(initial_positions, dtype=np.float64).copy()
  for _ in range(int(sd_steps)):
    e0, f = energy_fn.energy_and_forces(r)
    max_force = float(np.max(np.linalg.norm(f, axis=-1))) + 1e-8
    dt = min(max_displacement_per_step / max_force, dt_max)
    best_r, best_e = None, None
    for frac in (0.10, 0.25, 0.50, 1.00):  # the reference's selection order
      rt = r + frac * dt * f
      et = energy_fn(rt)
      if best_e is None or et < best_e:
        best_r, best_e = rt, et
    if best_e < e0:
      r = best_r
  return r


def run_simulation(system_params, initial_positions, temperature: float = 300.0,
                   min_steps: int = 500, therm_steps: int = 1000,
                   dielectric_constant: float = 1.0, implicit_solvent: bool = True,
                   solvent_dielectric: float = 78.5, solute_dielectric: float = 1.0,
                   key=None, sim_spec: SimulationSpec | None = None):
  """Minimise, thermalise, optionally run production (physics/simulate.py:357-508).

  Returns final positions (N, 3).
  """
  if not implicit_solvent:
    raise NotImplementedError("prolix_b200 implements the implicit-solvent path only")
  dt_ps, steps_prod = 2e-3, 0
  if sim_spec is not None:
    temperature = sim_spec.temperature
    dt_ps = sim_spec.dt
    steps_prod = sim_spec.steps
  sysd = system_to_dict(system_params)
  r0 = np.asarray(initial_positions, dtype=np.float64)
  sysd["positions"] = r0
  # the reference hands make_energy_fn a proxide Protein built from the
  # parameters (physics/simulate.py:400-414); here its 1-2 / 1-3 / 1-4
  # classes come from the bonds, as ExclusionSpec.from_protein derives them
  spec = None
  if "excl_pairs" not in sysd and sysd.get("excl_indices") is None:
    spec = exclusion_spec_from_bonds(sysd.get("bonds", np.zeros((0, 2))), r0.shape[0])
  efn = make_energy_fn(None, sysd, implicit_solvent=True, solvent_dielectric=solvent_dielectric,
                       solute_dielectric=solute_dielectric, exclusion_spec=spec)
  r = run_minimization(efn, r0, steps=min_steps)
  masses = np.asarray(sysd.get("masses", np.ones(r.shape[0])), dtype=np.float64)
  kT = BOLTZMANN_KCAL * temperature
  if key is None:
    key = np.array([0, 0], dtype=np.uint32)

  def langevin(r_start, n_steps, dt_ps_, gamma_ps):
    init_fn, apply_fn = nvt_langevin(efn, None, dt=dt_ps_ * 1000.0 / engine.AKMA_TIME_FS, kT=kT,
                                     gamma=engine.akma_gamma(gamma_ps), mass=masses)
    st = init_fn(key, r_start, mass=masses)
    if n_steps:
      st = apply_fn(st, n_steps)
    return st.position

  r = langevin(r, therm_steps, 2e-3, 1.0)
  if sim_spec is not None and steps_prod > 0:
    if sim_spec.ensemble == "nvt_langevin":
      return langevin(r, steps_prod, dt_ps, sim_spec.gamma)
    if sim_spec.ensemble == "nve":
      return langevin(r, steps_prod, dt_ps, 0.0)
    raise NotImplementedError(f"ensemble {sim_spec.ensemble!r} is outside the implicit-solvent "
                              "Langevin path built here")
  return r
