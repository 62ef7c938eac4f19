"""A ragged ensemble whose integrator state lives in host memory.

prolix's integrators are functional (``apply_fn(state) -> state``,
physics/settle.py:1698-1744): a caller that keeps the state on the host
between calls moves positions, momenta and forces across PCIe twice per
call.  ``StreamedEnsemble`` splits the systems into a few groups of
consecutive systems, each a ``Batch`` with its own CUDA stream, and steps
them with ``pb2_langevin_run_host``.  All groups share one stream for their
copies in and one for their copies out, so each direction moves one group's
state at a time at full PCIe speed, in group order, while other groups'
steps run: the transfers hide behind the arithmetic except for the first
group's copy in and the last group's copy out.  Each system's trajectory is
the one it has in any other batch (the pair kernels' sums do not depend on
the batch a system runs in).
"""

from __future__ import annotations

import numpy as np

from .engine import Batch


def partition(sizes, groups: int) -> list[tuple[int, int]]:
  """Ranges [a, b) of consecutive systems, at most ``groups`` of them, none
  empty, with about equal pair work (sum of n^2) each."""
  sizes = np.asarray(sizes, dtype=np.float64)
  if sizes.size == 0:
    raise ValueError("no systems")
  groups = max(1, min(int(groups), sizes.size))
  cum = np.cumsum(sizes * sizes)
  cuts = [0]
  for g in range(1, groups):
    c = int(np.searchsorted(cum, cum[-1] * g / groups, side="left")) + 1
    c = min(max(c, cuts[-1] + 1), sizes.size - (groups - g))
    cuts.append(c)
  cuts.append(sizes.size)
  return [(cuts[g], cuts[g + 1]) for g in range(groups)]


def pinned(shape, dtype=np.float64) -> np.ndarray:
  """A page-locked host array (host<->device copies from it are
  asynchronous and run at full PCIe speed)."""
  import torch
  t = torch.empty(shape, dtype=torch.from_numpy(np.zeros(0, dtype=dtype)).dtype, pin_memory=True)
  return t.numpy()


class StreamedEnsemble:
  """Systems in ``groups`` batches, each stepped on its own CUDA stream.

  State arrays are (n_atoms, 3) float64 in the order of ``systems``; use
  ``pinned`` arrays so that copies overlap computation.
  """

  def __init__(self, systems, groups: int = 12, device: int = 0, **batch_kw):
    import torch
    if isinstance(systems, dict):
      systems = [systems]
    sizes = [len(s["charges"]) for s in systems]
    self.ranges = partition(sizes, groups)
    self.batches = []
    try:
      for a, b in self.ranges:
        self.batches.append(Batch(systems[a:b], device=device, **batch_kw))
    except Exception:
      self.close()
      raise
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    self.atom_ranges = [(int(offs[a]), int(offs[b])) for a, b in self.ranges]
    self.n_atoms = int(offs[-1])
    self.n_systems = len(sizes)
    self.streams = [torch.cuda.Stream(device=device) for _ in self.batches]
    # one stream for every group's copies in and one for its copies out, so
    # that each direction moves one group's state at a time, in group order
    self.copy_in = torch.cuda.Stream(device=device)
    self.copy_out = torch.cuda.Stream(device=device)

  def _views(self, arr, g):
    a, b = self.atom_ranges[g]
    return arr[a:b]

  def synchronize(self):
    for s in (*self.streams, self.copy_in, self.copy_out):
      s.synchronize()

  def langevin_init(self):
    for bt, st in zip(self.batches, self.streams):
      bt.langevin_init(st.cuda_stream)

  def get_state(self, out=None, fields=("position", "momentum", "force")) -> dict:
    """The state of every system, gathered into ``out`` (allocated pinned
    when absent)."""
    out = dict(out or {})
    for f in fields:
      if f not in out:
        out[f] = pinned((self.n_atoms, 3))
    for g, (bt, st) in enumerate(zip(self.batches, self.streams)):
      bt.get_state(st.cuda_stream, fields=fields, out={f: self._views(out[f], g) for f in fields})
    return {f: out[f] for f in fields}

  def run_host(self, position, momentum, force, n_steps: int, wait: bool = True):
    """n_steps BAOAB steps of every system on the state in the three arrays,
    written back in place.  With ``wait`` it returns once all groups have
    finished; without, it returns at once, and a later call on the same
    arrays still reads each group's state only after that group's previous
    copy out has landed (the batch orders its copies), so a caller can queue
    several round trips and ``synchronize()`` before reading the arrays."""
    for a in (position, momentum, force):
      if not isinstance(a, np.ndarray) or a.shape != (self.n_atoms, 3):
        raise ValueError(f"run_host: arrays must be ({self.n_atoms}, 3)")
    for g, (bt, st) in enumerate(zip(self.batches, self.streams)):
      bt.langevin_run_host(self._views(position, g), self._views(momentum, g), self._views(force, g),
                           n_steps, st.cuda_stream, self.copy_in.cuda_stream, self.copy_out.cuda_stream)
    if wait:
      self.synchronize()

  def close(self):
    for bt in getattr(self, "batches", []):
      bt.close()
    self.batches = []

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()
