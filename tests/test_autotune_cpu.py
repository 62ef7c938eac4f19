"""Autotuner bookkeeping (bucket keys, cache) on the CPU with a stand-in batch."""

import numpy as np

from prolix_b200 import autotune


class FakeBatch:
  def __init__(self, sizes, cutoff=0.0):
    self.sizes = np.array(sizes)
    self.n_systems = len(sizes)
    self.n_atoms = int(self.sizes.sum())
    self.cutoff = cutoff
    self.seg = 8
    self.state = {"position": np.arange(6.0).reshape(2, 3), "momentum": np.ones((2, 3)),
                  "key": np.array([[1, 2]], dtype=np.uint32)}

    self.shapes = [(256, 3), (256, 2), (256, 2), (128, 3)]
    self.fuse = 1
    self.fblocks = 2

  def set_tile_segment(self, s):
    self.seg = s

  def block_shapes(self, p):
    return {0: [(256, 3), (128, 6)], 3: [(128, 3), (128, 2)]}.get(p, [(256, 2), (128, 4)])

  def set_force_blocks(self, n):
    self.fblocks = n

  def force_blocks(self):
    return self.fblocks

  def set_block_shape(self, p, t, m):
    self.shapes[p] = (t, m)

  def block_shape(self, p):
    return self.shapes[p]

  def set_fusion(self, f):
    self.fuse = f

  def fusion(self):
    return self.fuse

  def get_state(self):
    return {k: v.copy() for k, v in self.state.items()}

  def set_state(self, position=None, momentum=None, key=None):
    self.state = {"position": position, "momentum": momentum, "key": key}


def test_bucket_key_rounds_to_powers_of_two():
  a = autotune.bucket_key(FakeBatch([150, 3000]), "GPU")
  b = autotune.bucket_key(FakeBatch([200, 2800]), "GPU")
  c = autotune.bucket_key(FakeBatch([200, 2800], cutoff=9.0), "GPU")
  assert a == b != c


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
  monkeypatch.setenv("PROLIX_B200_TUNE_CACHE", str(tmp_path / "t.json"))
  cost = {2: 3.0, 4: 1.5, 8: 2.0}

  def timed(b, steps=4):
    # segment cost, minus a gain for a 128-thread force pass and for
    # fusion 3; everything else unchanged
    ms = cost[b.seg]
    if b.fblocks == 2 and b.shapes[1] == (128, 4):
      ms -= 0.2
    if b.fblocks == 4:
      ms -= 0.3 if b.shapes[3] == (128, 2) else 0.1
    if b.fuse == 3:
      ms -= 0.1
    return ms

  monkeypatch.setattr(autotune, "measure", lambda b, s, steps=4: (b.set_tile_segment(s), timed(b))[1])
  monkeypatch.setattr(autotune, "_time", timed)
  monkeypatch.setattr(autotune, "_gpu_name", lambda: "FAKE")
  fb = FakeBatch([100, 200])
  r = autotune.tune(fb, candidates=(2, 4, 8))
  assert r["segment"] == 4 and fb.seg == 4 and not r["cached"]
  # four i-blocks in the force pass at 128x2 (-0.3) beats two at 128x4 (-0.2)
  assert r["shapes"] == [[256, 3], [128, 4], [256, 2], [128, 2]] and fb.shapes[3] == (128, 2)
  assert r["force_blocks"] == 4 and fb.fblocks == 4
  assert r["fusion"] == 3 and fb.fuse == 3
  assert abs(r["ms"] - 1.1) < 1e-12
  fb2 = FakeBatch([100, 200])
  r2 = autotune.tune(fb2, candidates=(2, 4, 8))
  assert r2["cached"] and fb2.seg == 4 and fb2.shapes[3] == (128, 2) and fb2.fblocks == 4 and fb2.fuse == 3
