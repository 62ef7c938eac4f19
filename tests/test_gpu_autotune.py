"""Autotuner on the GPU: any tile segment gives bit-identical forces, and
tuning leaves the simulation state exactly as it was."""

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
