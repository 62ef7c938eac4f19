"""Trajectory records (prolix simulate.py:146-203, typing.py:652-707): the
msgpack payload of one frame and the length-prefixed file round trip."""

import numpy as np
import pytest

from prolix_b200 import trajectory as tr


def test_record_round_trip_drops_none():
  st = {"positions": np.arange(12, dtype=np.float32).reshape(4, 3),
        "velocities": np.full((4, 3), 0.5, np.float32), "step": 250, "time_ns": 0.0005,
        "potential_energy": None}
  d = tr.decode_record(tr.encode_record(st))
  assert set(d) == {"positions", "velocities", "step", "time_ns"}
  np.testing.assert_array_equal(d["positions"], st["positions"])
  assert d["positions"].dtype == np.float32 and d["step"] == 250


def test_file_round_trip(tmp_path):
  path = str(tmp_path / "t.pb2traj")
  frames = [{"positions": np.random.default_rng(k).normal(size=(5, 3)).astype(np.float32),
             "velocities": np.zeros((5, 3), np.float32), "step": 10 * k, "time_ns": 1e-5 * k}
            for k in range(7)]
  with tr.TrajectoryWriter(path) as w:
    w.write(frames[:3])
    for f in frames[3:]:
      w.write(f)
  back = list(tr.read_trajectory(path))
  assert [b["step"] for b in back] == [f["step"] for f in frames]
  for a, b in zip(frames, back):
    np.testing.assert_array_equal(a["positions"], b["positions"])
  bad = tmp_path / "bad"
  bad.write_bytes(b"nope")
  with pytest.raises(ValueError):
    list(tr.read_trajectory(str(bad)))
