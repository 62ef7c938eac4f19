"""Drop-in for prolix's production driver ``prolix.simulate.run_simulation``
(simulate.py:206-1113) on the implicit-solvent path.

Stages, as the reference runs them:

1. the energy at the start must be finite (:566-579);
2. FIRE minimisation in five stages of 500, 500, 500, 1000 and 3000 steps
   (:655-759).  The reference passes soft-core and restraint keywords to
   an energy function that ignores them (physics/system.py:229), so every
   stage minimises the standard energy.  Per stage it caps each atom's force
   at 10, 10, 100, 1000 and none, and caps displacements at 0.1 A per step
   except in the last stage.  It starts from the last stage's final
   positions, with dt_start = clip(0.001 / max |grad|, 1e-7, 0.001) and
   dt_max = min(10 dt_start, 0.01), both doubled (capped) after each stage;
3. gentle start (:833-880): 100 Langevin steps at dt/20, then 500 at dt/2,
   each from freshly drawn momenta, reverting to the minimised positions if
   a phase turns non-finite;
4. production: ``total_time_ns / save_interval_ns`` frames every
   ``save_interval_ns``, each with positions, velocities, potential and
   kinetic energy, written per epoch of ``accumulate_steps`` frames; a
   non-finite frame raises (:1050-1073);
5. returns the final state with its energy (:1098-1112).

Everything runs on the device batch; the trajectory file uses the record
layout of ``prolix_b200.trajectory``.  Deviation: the reference derives the
gentle-start keys from Python's string hash (randomised per process); here
they come from fixed offsets of the run's key.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import engine
from .system import system_to_dict
from .trajectory import TrajectoryWriter

BOLTZMANN_KCAL = engine.KB_KCAL
FIRE_STAGES = ((10.0, 500, True), (10.0, 500, True), (100.0, 500, True), (1000.0, 1000, True),
               (None, 3000, False))  # (force cap, steps, 0.1 A displacement cap)


@dataclasses.dataclass(frozen=True)
class PhysicsSpec:
  """prolix physics/spec.py:8-24 (implicit-solvent fields)."""
  dt: float = 2.0  # fs
  temperature_k: float = 300.0
  gamma: float = 1.0  # 1/ps

  @property
  def kT(self) -> float:
    return self.temperature_k * BOLTZMANN_KCAL


@dataclasses.dataclass
class SimulationSpec:
  """prolix simulate.py:60-139 (implicit-solvent fields)."""
  total_time_ns: float
  physics: PhysicsSpec = dataclasses.field(default_factory=PhysicsSpec)
  save_interval_ns: float = 0.001
  accumulate_steps: int = 500
  save_path: str = "trajectory.pb2traj"

  @property
  def step_size_fs(self) -> float:
    return self.physics.dt

  @property
  def temperature_k(self) -> float:
    return self.physics.temperature_k

  @property
  def gamma(self) -> float:
    return self.physics.gamma

  def __post_init__(self):
    if self.save_interval_ns <= 0:
      raise ValueError("save_interval_ns must be positive")
    if self.physics.dt <= 0:
      raise ValueError("step_size_fs must be positive")
    if self.accumulate_steps <= 0:
      raise ValueError("accumulate_steps must be positive")


@dataclasses.dataclass
class SimulationState:
  """prolix typing.py:652-669."""
  positions: np.ndarray
  velocities: np.ndarray
  step: int
  time_ns: float
  forces: np.ndarray | None = None
  mass: np.ndarray | None = None
  potential_energy: float | None = None
  kinetic_energy: float | None = None

  def numpy(self) -> dict:
    return dataclasses.asdict(self)


def _batch(sysd, positions, key, dt_fs, spec, device):
  return engine.Batch([dict(sysd, positions=positions, key=key, dt=engine.akma_dt(dt_fs),
                            kT=spec.physics.kT, gamma=engine.akma_gamma(spec.gamma))], device=device)


def minimize_fire_stages(sysd, positions, device=0, stages=FIRE_STAGES):
  """Stage 2 above; returns the minimised positions."""
  with engine.Batch([dict(sysd, positions=positions)], device=device) as b:
    e0, f0 = b.energy_forces()
    if not np.isfinite(e0[0][-1]):
      raise RuntimeError(f"Initial energy is non-finite ({e0[0][-1]:.2f} kcal/mol)")
    max_grad = float(np.max(np.linalg.norm(f0, axis=1)))
    dt_start = float(np.clip(0.001 / (max_grad + 1e-8), 1e-7, 0.001))
    dt_max = min(dt_start * 10.0, 0.01)
    b.min_setup()
    for cap, steps, disp in stages:
      b.min_fire(steps, k=0.0, dt_start=dt_start, dt_max=dt_max, max_disp=0.1 if disp else 0.0,
                 force_cap=cap or 0.0, keep_best=False)
      dt_start = min(dt_start * 2.0, 0.001)
      dt_max = min(dt_start * 10.0, 0.01)
    return b.get_state(fields=("position",))["position"].copy()


def run_simulation(system, initial_positions=None, spec: SimulationSpec | None = None, key=None,
                   device: int = 0, fire_stages=FIRE_STAGES) -> SimulationState:
  """prolix simulate.py:206-1113 for an implicit-solvent system dict."""
  if spec is None:
    raise ValueError("run_simulation needs a SimulationSpec")
  sysd = system_to_dict(system)
  r0 = np.asarray(initial_positions if initial_positions is not None else sysd["positions"], np.float64)
  masses = np.asarray(sysd.get("masses", np.full(r0.shape[0], 12.011)), np.float64)
  sysd = dict(sysd, masses=masses, origin=engine.default_origin(r0))
  k0, k1 = (0, 0) if key is None else (int(v) & 0xFFFFFFFF for v in np.asarray(key).reshape(2))

  r_min = minimize_fire_stages(sysd, r0, device, fire_stages)

  # gentle start: dt/20 then dt/2, fresh momenta each phase
  r_start = r_min
  for n, (scale, steps) in enumerate(((1.0 / 20.0, 100), (0.5, 500))):
    with _batch(sysd, r_start, (k0, (k1 + 101 * (n + 1)) & 0xFFFFFFFF), spec.step_size_fs * scale,
                spec, device) as b:
      b.langevin_init()
      b.langevin_run(steps)
      pos = b.get_state(fields=("position",))["position"]
    if not np.isfinite(pos).all():
      r_start = r_min
      break
    r_start = pos.copy()

  steps_per_save = round(spec.save_interval_ns * 1_000_000 / spec.step_size_fs)
  total_saves = int(spec.total_time_ns / spec.save_interval_ns)
  with _batch(sysd, r_start, (k0, k1), spec.step_size_fs, spec, device) as b, \
       TrajectoryWriter(spec.save_path) as writer:
    b.langevin_init()
    done = 0
    while done < total_saves:
      frames = []
      for _ in range(min(spec.accumulate_steps, total_saves - done)):
        b.langevin_run(steps_per_save)
        e, _ = b.energy_forces()
        st = b.get_state(fields=("position", "momentum"))
        if not np.isfinite(st["position"]).all():
          raise RuntimeError(f"Simulation instability detected: NaN/Inf positions at step "
                             f"{(done + len(frames) + 1) * steps_per_save}")
        p = st["momentum"]
        step = (done + len(frames) + 1) * steps_per_save
        frames.append({"positions": st["position"].astype(np.float32),
                       "velocities": (p / masses[:, None]).astype(np.float32),
                       "step": step, "time_ns": step * spec.step_size_fs * 1e-6,
                       "potential_energy": float(e[0][-1]),
                       "kinetic_energy": float(0.5 * np.sum(p ** 2 / masses[:, None]))})
      writer.write(frames)
      done += len(frames)
    e, f = b.energy_forces()
    st = b.get_state(fields=("position", "momentum"))
  p = st["momentum"]
  return SimulationState(positions=st["position"], velocities=p / masses[:, None],
                         step=total_saves * steps_per_save, time_ns=float(spec.total_time_ns), forces=f,
                         potential_energy=float(e[0][-1]),
                         kinetic_energy=float(0.5 * np.sum(p ** 2 / masses[:, None])))
