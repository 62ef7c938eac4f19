"""Trajectory output: the frames prolix's ``TrajectoryWriter`` stores
(simulate.py:146-203), streamed from a device ring buffer.

Each record is the msgpack payload of prolix ``SimulationState.numpy()``
(typing.py:652-707) for one system at one saved step: ``positions``,
``velocities`` (float32 (n, 3)), ``step`` and ``time_ns``.  Arrays use the
field layout of the msgpack-numpy encoding the reference uses ({"nd": True,
"type": dtype string, "kind", "shape", "data": bytes}); ``decode_record``
reads them back.  ArrayRecord (the reference's container) is not
available here; records go to a length-prefixed file: the magic bytes
``PB2TRAJ1`` then, per record, a little-endian uint32 length and the
payload.

``run_with_trajectory`` advances a batch in segments of ``save_interval``
steps and snapshots each frame into the device ring asynchronously; the
host fetches the ring once it is full (one synchronisation per ``capacity``
frames) and a background thread serialises and writes while the GPU runs
the next segments.

``XtcFrameSink`` (end of this file) is the reference's XTC sink; it takes
the same frames as ``TrajectoryWriter``.
"""

from __future__ import annotations

import queue
import struct
import threading

import msgpack
import numpy as np

MAGIC = b"PB2TRAJ1"


def _encode(obj):
  if isinstance(obj, np.ndarray):
    return {b"nd": True, b"type": obj.dtype.str, b"kind": b"", b"shape": list(obj.shape),
            b"data": obj.tobytes()}
  if isinstance(obj, np.generic):
    return obj.item()
  return obj


def _decode(obj):
  if isinstance(obj, dict) and obj.get(b"nd") is True:
    return np.frombuffer(obj[b"data"], dtype=np.dtype(obj[b"type"])).reshape(obj[b"shape"])
  return obj


def encode_record(state: dict) -> bytes:
  """msgpack bytes of one frame (None values dropped, as the reference does)."""
  return msgpack.packb({k: v for k, v in state.items() if v is not None}, default=_encode,
                       use_bin_type=True)


def decode_record(data: bytes) -> dict:
  out = msgpack.unpackb(data, object_hook=_decode, raw=False, strict_map_key=False)
  return {(k.decode() if isinstance(k, bytes) else k): v for k, v in out.items()}


class TrajectoryWriter:
  """Append-only frame file (see the module docstring for the layout)."""

  def __init__(self, path: str):
    self._f = open(path, "wb")
    self._f.write(MAGIC)
    self.closed = False
    self.count = 0

  def write(self, states):
    if self.closed:
      raise RuntimeError("Writer is closed")
    if isinstance(states, dict):
      states = [states]
    for st in states:
      payload = encode_record(st)
      self._f.write(struct.pack("<I", len(payload)))
      self._f.write(payload)
      self.count += 1

  def close(self):
    if not self.closed:
      self._f.close()
      self.closed = True

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()


def read_trajectory(path: str):
  """Yield the frames of a file written by TrajectoryWriter."""
  with open(path, "rb") as f:
    if f.read(len(MAGIC)) != MAGIC:
      raise ValueError(f"{path}: not a prolix_b200 trajectory")
    while True:
      head = f.read(4)
      if not head:
        return
      (n,) = struct.unpack("<I", head)
      yield decode_record(f.read(n))


def run_with_trajectory(batch, n_steps: int, save_interval: int, writers, capacity: int = 16,
                        dt_ns=None, stream=None) -> int:
  """Run ``n_steps`` Langevin steps of ``batch`` and save every
  ``save_interval`` steps.  ``writers``: one TrajectoryWriter or
  XtcFrameSink per system (or a single writer receiving every system's
  frames).  ``dt_ns``: per-system
  time step in ns for ``time_ns`` (default: the step count only).  Returns
  the number of frames saved per system."""
  if save_interval <= 0:
    raise ValueError("save_interval must be > 0")
  n_frames = n_steps // save_interval
  per_system = isinstance(writers, (list, tuple))
  if per_system and len(writers) != batch.n_systems:
    raise ValueError("one writer per system")
  batch.traj_setup(capacity)
  work: queue.Queue = queue.Queue(maxsize=2)
  err = []

  def drain():
    try:
      while True:
        item = work.get()
        if item is None:
          return
        pos, vel, steps = item
        for k in range(pos.shape[0]):
          for s in range(batch.n_systems):
            lo, hi = batch.offsets[s], batch.offsets[s + 1]
            step = int(steps[k, s])
            st = {"positions": pos[k, lo:hi], "velocities": vel[k, lo:hi], "step": step,
                  "time_ns": float(step * dt_ns[s]) if dt_ns is not None else None}
            (writers[s] if per_system else writers).write(st)
    except Exception as e:  # surfaced to the caller after the run
      err.append(e)

  t = threading.Thread(target=drain, daemon=True)
  t.start()
  try:
    slot = 0
    for _ in range(n_frames):
      batch.langevin_run(save_interval, stream)
      batch.traj_snapshot(slot, stream)
      slot += 1
      if slot == capacity:
        work.put(batch.traj_fetch(0, slot, stream))
        slot = 0
    if slot:
      work.put(batch.traj_fetch(0, slot, stream))
    rest = n_steps - n_frames * save_interval
    if rest:
      batch.langevin_run(rest, stream)
  finally:
    work.put(None)
    t.join()
  if err:
    raise err[0]
  return n_frames


# --- XTC sink (prolix api/xtc_sink.py:1-140) ---------------------------------
#
# The reference writes XTC through mdtraj's XTCTrajectoryFile (Å in, nm on
# disk, time in ps) behind a small backend protocol so another writer can be
# swapped in.  The same surface here: ``XtcFrameSink`` takes (n_atoms, 3) or
# (n_frames, n_atoms, 3) positions in Å, and also accepts the frame dicts of
# ``run_with_trajectory`` through ``write``, so device-ring frames stream
# straight into an XTC file.  The XTC codec itself is mdtraj's; without mdtraj
# the default backend raises ImportError when the sink is created.

ANGSTROM_PER_NM = 10.0


class XtcWriterBackend:
  """Frame writer protocol (xtc_sink.py:30-38): ``write_frame(coords_angstrom,
  *, time_ps=0.0)`` appends one (n_atoms, 3) frame; ``close()`` flushes."""

  def write_frame(self, coords_angstrom, *, time_ps: float = 0.0) -> None:
    raise NotImplementedError

  def close(self) -> None:
    raise NotImplementedError


class MdtrajXtcWriter(XtcWriterBackend):
  """XTC through mdtraj (xtc_sink.py:41-75): Å in, nm on disk."""

  def __init__(self, path):
    try:
      from mdtraj.formats import XTCTrajectoryFile
    except ImportError as e:
      raise ImportError("XTC output needs mdtraj (the XTC codec the reference uses); "
                        "pass another XtcWriterBackend or install mdtraj") from e
    import os
    self.path = str(path)
    os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
    self._file = XTCTrajectoryFile(self.path, "w")
    self._closed = False

  def write_frame(self, coords_angstrom, *, time_ps: float = 0.0) -> None:
    if self._closed:
      raise RuntimeError(f"XTC writer already closed: {self.path}")
    coords = np.asarray(coords_angstrom, dtype=np.float32)
    if coords.ndim != 2 or coords.shape[1] != 3:
      raise ValueError(f"expected (n_atoms, 3), got {coords.shape}")
    self._file.write(coords[np.newaxis] / ANGSTROM_PER_NM,
                     time=np.asarray([time_ps], dtype=np.float32))

  def close(self) -> None:
    if not self._closed:
      self._file.close()
      self._closed = True


class XtcFrameSink:
  """Positions → XTC frames (xtc_sink.py:78-121).  ``ordered`` is always
  True: frames are written in call order.  Called directly, frame k gets
  ``time_ps = k`` as in the reference; frames arriving through ``write``
  (the ``run_with_trajectory`` writer interface) carry their own
  ``time_ns`` when it is set, converted to ps."""

  ordered = True

  def __init__(self, path, backend: XtcWriterBackend | None = None):
    self.path = str(path)
    self._owns_backend = backend is None
    self.backend = MdtrajXtcWriter(self.path) if backend is None else backend
    self.count = 0
    self.closed = False

  def _frame(self, coords, time_ps) -> None:
    if self.closed:
      raise RuntimeError("Writer is closed")
    self.backend.write_frame(coords, time_ps=float(self.count if time_ps is None else time_ps))
    self.count += 1

  def __call__(self, x) -> None:
    arr = np.asarray(x, dtype=np.float32)
    if arr.ndim == 2:
      arr = arr[np.newaxis]
    if arr.ndim != 3 or arr.shape[-1] != 3:
      raise ValueError(f"XtcFrameSink expected 2D or 3D positions, got {arr.shape}")
    for frame in arr:
      self._frame(frame, None)

  def write(self, states) -> None:
    if isinstance(states, dict):
      states = [states]
    for st in states:
      pos = np.asarray(st["positions"], dtype=np.float32)
      if pos.ndim != 2 or pos.shape[1] != 3:
        raise ValueError(f"expected (n_atoms, 3) positions, got {pos.shape}")
      t = st.get("time_ns")
      self._frame(pos, None if t is None else float(t) * 1e3)

  def close(self) -> None:
    if not self.closed:
      if self._owns_backend:
        self.backend.close()
      self.closed = True

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()


def write_positions_xtc(path, positions_angstrom, *, backend: XtcWriterBackend | None = None):
  """Write (n_frames, n_atoms, 3) or (n_atoms, 3) positions in Å to an XTC
  file and return its path (xtc_sink.py:124-140)."""
  sink = XtcFrameSink(path, backend=backend)
  try:
    sink(positions_angstrom)
  finally:
    sink.close()
  return path
