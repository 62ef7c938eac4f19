"""Batched minimisation on the GPU (pb2_min_*) against the FP64 restatement
(oracle/minimize.py): restrained steepest descent and FIRE trajectories,
per-system independence in a ragged batch, and the full staged protocol of
prolix ``batched_minimize``."""

import numpy as np
import pytest

from oracle import energy as oenergy
from oracle import minimize as om
from prolix_b200 import engine, synth
from prolix_b200.minimize import batched_minimize

pytestmark = pytest.mark.gpu


def _sys(n, seed):
  s = synth.make_chain(n, seed, compact=True, **synth.PHYSICAL_RANGES)
  return dict(s, origin=engine.default_origin(s["positions"]))


def test_steepest_descent_matches_oracle():
  s = _sys(166, 11)
  heavy = np.asarray(s["masses"]) > 1.1
  with engine.Batch([s]) as b:
    b.min_setup()
    b.min_sd(25, k=500.0, kind="heavy", dt=0.002, max_dx=0.01)
    got = b.get_state(fields=("position",))["position"]
  ref = om.steepest_descent(s, s["positions"], s["positions"], heavy.astype(float), 25, 500.0, 0.002, 0.01)
  assert np.max(np.abs(got - ref)) < 1e-5
  assert np.max(np.abs(got - s["positions"])) > 1e-3  # it moved


def test_fire_matches_oracle_and_is_independent_of_the_batch():
  s, other = _sys(166, 12), _sys(300, 13)
  heavy = (np.asarray(s["masses"]) > 1.1).astype(float)
  args = dict(k=125.0, kind="backbone", dt_start=1e-3, dt_max=1e-2, max_disp=0.1)
  with engine.Batch([s]) as b:
    b.min_setup()
    b.min_fire(40, **args)
    alone = b.get_state(fields=("position",))["position"]
  with engine.Batch([other, s]) as b:
    b.min_setup()
    b.min_fire(40, **args)
    mixed = b.split(b.get_state(fields=("position",))["position"])[1]
  np.testing.assert_array_equal(mixed, alone)
  best, _ = om.fire(s, s["positions"], s["positions"], heavy, s["masses"], 40, 125.0, 1e-3, 1e-2, 0.1)
  assert np.max(np.abs(alone - best)) < 1e-5
  assert np.max(np.abs(alone - s["positions"])) > 1e-4


def test_batched_minimize_lowers_energy_and_force():
  systems = [_sys(n, 20 + i) for i, n in enumerate((166, 420, 900))]
  with engine.Batch(systems) as b:
    b.min_setup()
    rms0 = b.min_rms()
  pos, converged, rms = batched_minimize(systems, max_steps=300, fire_stage_steps=(150, 150, 150, 300))
  assert converged.shape == (3,) and rms.shape == (3,)
  assert np.all(rms < 0.5 * rms0)
  for s, p in zip(systems, pos):
    assert np.isfinite(p).all()
    assert oenergy.total_energy(s, p) < oenergy.total_energy(s, s["positions"])


def test_fire_force_cap_final_state_matches_oracle():
  # prolix.simulate's stages: per-atom force cap on the first half kick, no
  # displacement cap, the stage ends at its final positions
  s = _sys(166, 14)
  with engine.Batch([s]) as b:
    b.min_setup()
    b.min_fire(40, dt_start=1e-3, dt_max=1e-2, max_disp=0.0, force_cap=10.0, keep_best=False)
    got = b.get_state(fields=("position",))["position"]
  _, final = om.fire(s, s["positions"], s["positions"], np.zeros(166), s["masses"], 40, 0.0, 1e-3, 1e-2,
                     0.0, force_cap=10.0)
  assert np.max(np.abs(got - final)) < 1e-5


def test_production_run_simulation(tmp_path):
  from prolix_b200 import production, trajectory
  s = _sys(166, 15)
  spec = production.SimulationSpec(total_time_ns=0.002, save_interval_ns=0.0005, accumulate_steps=3,
                                   save_path=str(tmp_path / "prod.pb2traj"),
                                   physics=production.PhysicsSpec(dt=2.0))
  stages = ((10.0, 100, True), (100.0, 100, True), (None, 200, False))
  final = production.run_simulation(s, s["positions"], spec, key=(0, 9), fire_stages=stages)
  frames = list(trajectory.read_trajectory(spec.save_path))
  assert [f["step"] for f in frames] == [250, 500, 750, 1000]
  assert all(np.isfinite(f["potential_energy"]) and f["kinetic_energy"] > 0 for f in frames)
  assert final.step == 1000 and np.isfinite(final.positions).all()
  np.testing.assert_array_equal(frames[-1]["positions"], final.positions.astype(np.float32))


def test_lbfgs_polish_matches_oracle_and_descends():
  s = _sys(166, 16)
  with engine.Batch([s]) as b:
    b.min_setup()
    b.min_lbfgs(3, tol=1e-6, max_step=0.1, hist=10)
    got = b.get_state(fields=("position",))["position"]
  ref = om.lbfgs(s, s["positions"], 3, tol=1e-6, max_step=0.1, hist=10)
  assert np.max(np.abs(got - ref)) < 1e-5
  assert np.max(np.abs(got - s["positions"])) > 1e-4
  # a longer polish lowers energy and gradient (Armijo steps)
  with engine.Batch([s]) as b:
    b.min_setup()
    e0, f0 = b.energy_forces()
    conv = b.min_lbfgs(60, tol=1e-6, max_step=0.1, hist=10)
    e1, f1 = b.energy_forces()
  assert conv.shape == (1,)
  assert e1[0][-1] < e0[0][-1] and np.linalg.norm(f1) < np.linalg.norm(f0)


def test_batched_minimize_with_lbfgs_polish():
  systems = [_sys(n, 40 + i) for i, n in enumerate((166, 300))]
  _, _, rms_fire = batched_minimize(systems, max_steps=100, lbfgs_steps=0,
                                    fire_stage_steps=(50, 50, 50, 100))
  pos, converged, rms = batched_minimize(systems, max_steps=100, lbfgs_steps=100,
                                         fire_stage_steps=(50, 50, 50, 100))
  assert np.all(rms < rms_fire)
  assert all(np.isfinite(p).all() for p in pos)
