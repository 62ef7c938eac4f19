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


class _StubXtc(tr.XtcWriterBackend):
  def __init__(self):
    self.frames, self.times, self.closed = [], [], False

  def write_frame(self, coords_angstrom, *, time_ps=0.0):
    self.frames.append(np.array(coords_angstrom))
    self.times.append(time_ps)

  def close(self):
    self.closed = True


def _tiny_traj():
  return np.array([[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]],
                   [[0.1, 0.0, 0.0], [1.1, 0.0, 0.0], [0.0, 1.1, 0.0]]], dtype=np.float32)


def test_xtc_sink_frames_in_order_with_frame_index_times():
  """xtc_sink.py:96-111: 2D or 3D positions in Å, one backend frame each,
  time_ps = running frame index; a given backend is not closed by the sink."""
  be = _StubXtc()
  traj = _tiny_traj()
  with tr.XtcFrameSink("unused.xtc", backend=be) as sink:
    assert sink.ordered is True
    sink(traj)
    sink(traj[0].astype(np.float64))
  assert be.times == [0.0, 1.0, 2.0] and not be.closed
  for got, want in zip(be.frames, [traj[0], traj[1], traj[0]]):
    assert got.dtype == np.float32 and got.shape == (3, 3)
    np.testing.assert_array_equal(got, want)
  with pytest.raises(ValueError):
    tr.XtcFrameSink("unused.xtc", backend=_StubXtc())(np.zeros(3))
  with pytest.raises(ValueError):
    tr.XtcFrameSink("unused.xtc", backend=_StubXtc())(np.zeros((2, 4, 2)))


def test_xtc_sink_takes_trajectory_frames():
  """The run_with_trajectory writer interface: frame dicts, time from
  time_ns (ns → ps) when set, else the frame index."""
  be = _StubXtc()
  sink = tr.XtcFrameSink("unused.xtc", backend=be)
  pos = np.arange(12, dtype=np.float32).reshape(4, 3)
  sink.write({"positions": pos, "velocities": pos, "step": 5, "time_ns": 0.002})
  sink.write([{"positions": pos + 1, "step": 10, "time_ns": None}])
  np.testing.assert_allclose(be.times, [2.0, 1.0])
  np.testing.assert_array_equal(be.frames[1], pos + 1)
  sink.close()
  with pytest.raises(RuntimeError):
    sink.write({"positions": pos})


def test_write_positions_xtc_and_missing_codec(tmp_path):
  be = _StubXtc()
  out = tr.write_positions_xtc(tmp_path / "t.xtc", _tiny_traj(), backend=be)
  assert out == tmp_path / "t.xtc" and len(be.frames) == 2
  try:
    import mdtraj  # noqa: F401
  except ImportError:
    with pytest.raises(ImportError, match="mdtraj"):
      tr.XtcFrameSink(tmp_path / "u.xtc")
