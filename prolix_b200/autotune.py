"""Autotuner for the pair kernels' work shapes and the step's schedule.

Three knobs, tuned in turn, each by timing a few full MD steps per
candidate (CUDA events on the launching stream; the fastest wins):

* ``tile_segment``: 32 x 32 tiles per work item.  Short items balance the
  dynamically scheduled passes better, long items amortise loading a
  warp's i-block.
* the block shape of each pair pass (threads per block, resident blocks
  per SM the registers are sized for), among the shapes compiled for it
  (``Batch.block_shapes``): more, smaller blocks against fewer registers
  per thread; and for the force pass, two or four i-blocks per warp (four
  share each j atom's loads, at more registers), each with its shapes.
* fusion (``_lib.FUSE_*``): the bonded terms as the chain pass's tail work,
  and the Born radii finalized as the descreening pass's tail work (one
  chunk per 32-atom block, started once its system's items are summed),
  against launches of their own.

The best choice depends on the size mix of the batch; it is cached in JSON
keyed by GPU name and a workload bucket (number of systems, total atoms,
largest system, cutoff mode, each rounded to a power of two).  The batch's
state is snapshotted before tuning and restored after, so tuning does not
advance the simulation.

Cache file: ``$PROLIX_B200_TUNE_CACHE`` or ~/.cache/prolix_b200/autotune.json.
"""

from __future__ import annotations

import json
import math
import os
from pathlib import Path

import numpy as np

CANDIDATES = (2, 4, 8, 16, 32)


def cache_path() -> Path:
  env = os.environ.get("PROLIX_B200_TUNE_CACHE")
  if env:
    return Path(env)
  return Path.home() / ".cache" / "prolix_b200" / "autotune.json"


def _p2(x: float) -> int:
  return 1 << max(0, int(math.ceil(math.log2(max(1.0, float(x))))))


def bucket_key(batch, gpu_name: str) -> str:
  return "|".join([gpu_name, f"sys{_p2(batch.n_systems)}", f"atoms{_p2(batch.n_atoms)}",
                   f"nmax{_p2(int(batch.sizes.max()))}",
                   "cut" if getattr(batch, "cutoff", 0.0) > 0 else "all"])


def _load(path: Path) -> dict:
  try:
    return json.loads(path.read_text())
  except (OSError, ValueError):
    return {}


def _store(path: Path, data: dict):
  path.parent.mkdir(parents=True, exist_ok=True)
  tmp = path.with_suffix(".tmp")
  tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
  os.replace(tmp, path)


def _gpu_name() -> str:
  try:
    import torch
    return torch.cuda.get_device_name(0).replace(" ", "_")
  except Exception:
    return "unknown_gpu"


def _time(batch, steps: int) -> float:
  """Mean ms per MD step of ``batch`` as it is configured now."""
  import torch
  stream = torch.cuda.current_stream().cuda_stream
  batch.langevin_run(1, stream)  # capture
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  torch.cuda.synchronize()
  e0.record()
  batch.langevin_run(steps, stream)
  e1.record()
  torch.cuda.synchronize()
  return e0.elapsed_time(e1) / steps


def measure(batch, segment: int, steps: int = 4) -> float:
  """Mean ms per MD step of ``batch`` with ``segment`` tiles per item."""
  batch.set_tile_segment(segment)
  return _time(batch, steps)


def apply(batch, choice: dict):
  """Set a tuned (or cached) choice on the batch."""
  batch.set_tile_segment(int(choice["segment"]))
  for p, shape in enumerate(choice.get("shapes") or []):
    batch.set_block_shape(p, int(shape[0]), int(shape[1]))
  if choice.get("force_blocks") is not None:
    batch.set_force_blocks(int(choice["force_blocks"]))
  if choice.get("fusion") is not None:
    batch.set_fusion(int(choice["fusion"]))


def tune(batch, candidates=CANDIDATES, steps: int = 4, use_cache: bool = True,
         shapes: bool = True, fusion: bool = True) -> dict:
  """Pick ``tile_segment``, then each pair pass's block shape, then the
  fusion flags for ``batch`` (set on the batch) and return {"segment",
  "shapes", "fusion", "ms", "timings", "cached", "key"}."""
  key = bucket_key(batch, _gpu_name())
  path = cache_path()
  data = _load(path) if use_cache else {}
  if use_cache and key in data and "force_blocks" in data[key]:
    apply(batch, data[key])
    return {**data[key], "cached": True, "key": key}
  snap = batch.get_state()
  timings = {}
  for c in candidates:
    timings[f"segment={c}"] = measure(batch, c, steps)
  best_seg = min(candidates, key=lambda c: timings[f"segment={c}"])
  batch.set_tile_segment(int(best_seg))
  best_ms = timings[f"segment={best_seg}"]
  chosen_shapes = [list(batch.block_shape(p)) for p in range(4)]
  chosen_blocks = batch.force_blocks()
  if shapes:
    for p in range(3):
      for t, m in batch.block_shapes(p):
        if [t, m] == chosen_shapes[p]:
          continue
        batch.set_block_shape(p, t, m)
        ms = _time(batch, steps)
        timings[f"pass{p}={t}x{m}"] = ms
        if ms < best_ms:
          best_ms = ms
          chosen_shapes[p] = [t, m]
        batch.set_block_shape(p, *chosen_shapes[p])
    # the force pass with four i-blocks per warp, in each of its shapes
    # (without a pair list: with one, the force pass keeps two)
    batch.set_force_blocks(4)
    for t, m in batch.block_shapes(3):
      batch.set_block_shape(3, t, m)
      ms = _time(batch, steps)
      timings[f"force4={t}x{m}"] = ms
      if ms < best_ms:
        best_ms = ms
        chosen_shapes[3] = [t, m]
        chosen_blocks = 4
    batch.set_block_shape(3, *chosen_shapes[3])
    batch.set_force_blocks(chosen_blocks)
  chosen_fusion = batch.fusion()
  if fusion:
    for f in range(4):
      if f == chosen_fusion:
        continue
      batch.set_fusion(f)
      ms = _time(batch, steps)
      timings[f"fusion={f}"] = ms
      if ms < best_ms:
        best_ms = ms
        chosen_fusion = f
      batch.set_fusion(chosen_fusion)
  batch.set_state(position=snap["position"], momentum=snap["momentum"], key=snap["key"])
  result = {"segment": int(best_seg), "shapes": chosen_shapes, "force_blocks": int(chosen_blocks),
            "fusion": int(chosen_fusion), "ms": best_ms, "timings": timings}
  if use_cache:
    data[key] = result
    _store(path, data)
  return {**result, "cached": False, "key": key}
