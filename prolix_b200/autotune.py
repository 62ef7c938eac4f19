"""Autotuner for the pair kernels' work-item shape.

The knob is the number of 32 x 32 tiles per work item (``tile_segment``):
short items balance the dynamically scheduled passes better, long items
amortise loading a warp's i-block.  The best value depends on the size mix
of the batch, so it is measured: each candidate runs a few full MD steps
(CUDA events on the launching stream), the fastest wins, and the choice is
cached in JSON keyed by GPU name and a workload bucket (number of systems,
total atoms, largest system, cutoff mode, each rounded to a power of two).
The batch's state is snapshotted before tuning and restored after, so
tuning does not advance the simulation.

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


def measure(batch, segment: int, steps: int = 4) -> float:
  """Mean ms per MD step of ``batch`` with ``segment`` tiles per item."""
  import torch
  batch.set_tile_segment(segment)
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


def tune(batch, candidates=CANDIDATES, steps: int = 4, use_cache: bool = True) -> dict:
  """Pick ``tile_segment`` for ``batch`` (set on the batch) and return
  {"segment", "ms", "timings", "cached", "key"}."""
  key = bucket_key(batch, _gpu_name())
  path = cache_path()
  data = _load(path) if use_cache else {}
  if use_cache and key in data:
    seg = int(data[key]["segment"])
    batch.set_tile_segment(seg)
    return {"segment": seg, "ms": data[key].get("ms"), "timings": data[key].get("timings"),
            "cached": True, "key": key}
  snap = batch.get_state()
  timings = {}
  for c in candidates:
    timings[str(c)] = measure(batch, c, steps)
  best = min(timings, key=timings.get)
  batch.set_tile_segment(int(best))
  batch.set_state(position=snap["position"], momentum=snap["momentum"], key=snap["key"])
  result = {"segment": int(best), "ms": timings[best], "timings": timings}
  if use_cache:
    data[key] = result
    _store(path, data)
  return {**result, "cached": False, "key": key}
