"""Trajectory frames from the device ring (pb2_traj_*) through
run_with_trajectory: frame count across ring wrap-around, saved steps, and
frames equal to the state at those steps."""

import numpy as np
import pytest

from oracle import prng
from prolix_b200 import engine, synth
from prolix_b200 import trajectory as tr

pytestmark = pytest.mark.gpu


def test_streamed_frames_match_the_state(tmp_path):
  systems = [synth.make_chain(n, 90 + n, compact=True, **synth.PHYSICAL_RANGES) for n in (166, 230)]
  paths = [str(tmp_path / f"s{k}.pb2traj") for k in range(2)]
  with engine.Batch(systems, key=prng.prng_key(3)) as b:
    b.langevin_init()
    writers = [tr.TrajectoryWriter(p) for p in paths]
    n = tr.run_with_trajectory(b, 33, 5, writers, capacity=4, dt_ns=[1e-6, 1e-6])
    for w in writers:
      w.close()
    st = b.get_state()
  assert n == 6
  masses = [np.asarray(s["masses"])[:, None] for s in systems]
  for k, p in enumerate(paths):
    frames = list(tr.read_trajectory(p))
    assert [f["step"] for f in frames] == [5, 10, 15, 20, 25, 30]
    assert frames[-1]["time_ns"] == pytest.approx(30e-6)
    assert frames[0]["positions"].shape == (len(systems[k]["charges"]), 3)
  # replay the same run without saving: the last frame is the state at step 30
  with engine.Batch(systems, key=prng.prng_key(3)) as b:
    b.langevin_init()
    b.langevin_run(30)
    st30 = b.get_state()
  for k, p in enumerate(paths):
    last = list(tr.read_trajectory(p))[-1]
    lo, hi = b.offsets[k], b.offsets[k + 1]
    np.testing.assert_array_equal(last["positions"], st30["position"][lo:hi].astype(np.float32))
    np.testing.assert_array_equal(last["velocities"],
                                  (st30["momentum"][lo:hi] * (1.0 / masses[k])).astype(np.float32))
  assert st["step"][0] == 33


class _Frames(tr.XtcWriterBackend):
  def __init__(self):
    self.frames, self.times = [], []

  def write_frame(self, coords_angstrom, *, time_ps=0.0):
    self.frames.append(np.array(coords_angstrom))
    self.times.append(time_ps)

  def close(self):
    pass


def test_xtc_sink_gets_the_ring_frames(tmp_path):
  """XtcFrameSink as the run_with_trajectory writer: the same positions as
  the msgpack records of an identical run, with time in ps."""
  systems = [synth.make_chain(n, 40 + n, compact=True, **synth.PHYSICAL_RANGES) for n in (150, 201)]
  paths = [str(tmp_path / f"s{k}.pb2traj") for k in range(2)]
  with engine.Batch(systems, key=prng.prng_key(8)) as b:
    b.langevin_init()
    writers = [tr.TrajectoryWriter(p) for p in paths]
    tr.run_with_trajectory(b, 20, 4, writers, capacity=3, dt_ns=[1e-6, 2e-6])
    for w in writers:
      w.close()
  backends = [_Frames(), _Frames()]
  with engine.Batch(systems, key=prng.prng_key(8)) as b:
    b.langevin_init()
    sinks = [tr.XtcFrameSink(tmp_path / f"s{k}.xtc", backend=be) for k, be in enumerate(backends)]
    assert tr.run_with_trajectory(b, 20, 4, sinks, capacity=3, dt_ns=[1e-6, 2e-6]) == 5
  for k, (p, be) in enumerate(zip(paths, backends)):
    frames = list(tr.read_trajectory(p))
    assert len(be.frames) == len(frames) == 5
    np.testing.assert_allclose(be.times, [4e-3 * (k + 1) * (f + 1) for f in range(5)], rtol=1e-12)
    for f, got in zip(frames, be.frames):
      np.testing.assert_array_equal(got, f["positions"])
