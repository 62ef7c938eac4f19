"""Replica exchange on the GPU: the device permutation of whole systems
(pb2_permute_systems) and a short parallel-tempering run."""

import numpy as np
import pytest

from oracle import prng
from prolix_b200 import engine, synth
from prolix_b200 import replica_exchange as rx

pytestmark = pytest.mark.gpu


def test_permute_systems_moves_whole_states():
  s = synth.make_chain(166, 31, compact=True, **synth.PHYSICAL_RANGES)
  origin = engine.default_origin(s["positions"])
  reps = [dict(s, origin=origin, key=prng.prng_key(40 + i), kT=engine.KB_KCAL * t)
          for i, t in enumerate((300.0, 330.0, 360.0))]
  with engine.Batch(reps) as b:
    b.langevin_init()
    b.langevin_run(20)
    st0 = b.get_state()
    perm = np.array([2, 0, 1])
    b.permute_systems(perm)
    st1 = b.get_state()
    for f in ("position", "momentum", "force"):
      old, new = b.split(st0[f]), b.split(st1[f])
      for slot in range(3):
        np.testing.assert_array_equal(new[slot], old[perm[slot]])
    np.testing.assert_array_equal(st1["key"], st0["key"])  # keys stay with the slots
    b.permute_systems(np.argsort(perm))
    st2 = b.get_state()
    for f in ("position", "momentum", "force"):
      np.testing.assert_array_equal(st2[f], st0[f])
    b.langevin_run(5)
    assert np.isfinite(b.get_state()["position"]).all()
    with pytest.raises(Exception):
      b.permute_systems(np.array([0, 0, 1]))


def test_permute_systems_between_different_stored_orders():
  # replicas created from different structures store their atoms in
  # different spatial orders; a swap still moves each atom's state to the
  # same atom of the other slot
  s = synth.make_chain(300, 32, compact=True, **synth.PHYSICAL_RANGES)
  rng = np.random.default_rng(5)
  pos2 = s["positions"] + rng.normal(0.0, 0.4, s["positions"].shape)
  origin = engine.default_origin(s["positions"])
  reps = [dict(s, origin=origin, key=prng.prng_key(60)), dict(s, positions=pos2, origin=origin,
                                                              key=prng.prng_key(61))]
  with engine.Batch(reps) as b:
    b.langevin_init()
    st0 = b.get_state()
    b.permute_systems(np.array([1, 0]))
    st1 = b.get_state()
    for f in ("position", "momentum", "force"):
      old, new = b.split(st0[f]), b.split(st1[f])
      np.testing.assert_array_equal(new[0], old[1])
      np.testing.assert_array_equal(new[1], old[0])
    # the forces the swap carried are the forces at the swapped positions
    e, f = b.energy_forces()
    assert np.linalg.norm(f - st1["force"]) / np.linalg.norm(f) < 1e-6


def test_short_parallel_tempering_run():
  s = synth.make_chain(166, 32, compact=True, **synth.PHYSICAL_RANGES)
  spec = rx.ReplicaExchangeSpec(n_replicas=4, min_temp=300.0, max_temp=450.0, step_size_fs=1.0,
                                exchange_interval_ps=0.05)
  st = rx.run_replica_exchange(s, s["positions"], spec, key=(0, 5), n_intervals=8)
  assert sorted(st.walker_indices.tolist()) == [0, 1, 2, 3]
  assert st.step == 8 * 50
  assert st.exchange_attempts >= 8 and st.exchange_successes <= st.exchange_attempts
  assert np.isfinite(st.positions).all() and np.isfinite(st.potential_energy).all()
  assert st.positions.shape == (4, 166, 3)
