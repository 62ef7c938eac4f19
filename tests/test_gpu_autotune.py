"""Autotuner on the GPU: any tile segment, block shape or fusion choice
gives bit-identical forces and steps, and tuning leaves the simulation
state exactly as it was."""

import numpy as np
import pytest

from prolix_b200 import autotune, engine, synth

pytestmark = pytest.mark.gpu


def _systems():
  return [synth.make_chain(n, 700 + k, compact=True) for k, n in enumerate([150, 900, 2100, 64])]


def test_forces_independent_of_tile_segment():
  with engine.Batch(_systems()) as b:
    ref = b.forces()
    for seg in (1, 3, 8, 32):
      b.set_tile_segment(seg)
      assert b.tile_segment() == seg
      np.testing.assert_array_equal(b.forces(), ref)


def test_block_shapes_and_fusion_leave_results_bitwise_equal():
  from oracle import energy as oenergy
  systems = _systems()
  fields = ("position", "momentum", "force")
  with engine.Batch(systems) as b:
    ref = b.forces()
    b.langevin_init()
    b.langevin_run(7)
    ref_st = b.get_state(fields=fields)
  for p in range(3):
    with engine.Batch(systems) as b:
      for t, m in b.block_shapes(p):
        b.set_block_shape(p, t, m)
        assert b.block_shape(p) == (t, m)
        np.testing.assert_array_equal(b.forces(), ref)
  with engine.Batch(systems) as b:
    b.set_force_blocks(4)
    assert b.force_blocks() == 4
    for t, m in b.block_shapes(3):
      b.set_block_shape(3, t, m)
      assert b.block_shape(3) == (t, m)
      np.testing.assert_array_equal(b.forces(), ref)
  for f in range(4):
    with engine.Batch(systems) as b:
      b.set_fusion(f)
      assert b.fusion() == f
      b.langevin_init()
      b.langevin_run(7)
      st = b.get_state(fields=fields)
      for k in fields:
        np.testing.assert_array_equal(st[k], ref_st[k])
  # and the tuned choice matches the oracle
  s = systems[1]
  e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"])
  with engine.Batch([s]) as b:
    autotune.tune(b, candidates=(4, 16), steps=2, use_cache=False)
    f = b.forces()
  assert np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref) < 1e-5


def test_tune_restores_state_and_caches(tmp_path, monkeypatch):
  monkeypatch.setenv("PROLIX_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
  with engine.Batch(_systems()) as b:
    b.langevin_init()
    b.langevin_run(3)
    before = b.get_state()
    res = autotune.tune(b, candidates=(2, 8), steps=2)
    after = b.get_state()
    assert res["segment"] in (2, 8) and not res["cached"]
    assert b.tile_segment() == res["segment"]
    for k in ("position", "momentum", "key"):
      np.testing.assert_array_equal(before[k], after[k])
    res2 = autotune.tune(b, candidates=(2, 8), steps=2)
    assert res2["cached"] and res2["segment"] == res["segment"]


@pytest.mark.parametrize("cutoff", [0.0, 9.0])
def test_four_block_force_kernel_equals_the_two_block_one(cutoff):
  # ragged sizes (one atom, one block, partial blocks, i-block counts not
  # multiples of 4), exclusions and 1-4 pairs, with and without a cutoff
  # (no pair list, so the four-block kernel runs): forces and trajectories
  # are the same bit for bit
  sizes = [1, 2, 20, 31, 32, 33, 64, 97, 128, 129, 130, 160, 193, 260, 1000]
  systems = [synth.make_chain(n, 40 + k, compact=True) for k, n in enumerate(sizes)]
  out = {}
  for blocks in (2, 4):
    with engine.Batch(systems, cutoff=cutoff, pair_list=False) as b:
      b.set_force_blocks(blocks)
      f = b.forces()
      b.langevin_init()
      b.langevin_run(5)
      out[blocks] = (f, b.get_state(fields=("position", "momentum")))
  np.testing.assert_array_equal(out[2][0], out[4][0])
  for k in ("position", "momentum"):
    np.testing.assert_array_equal(out[2][1][k], out[4][1][k])
