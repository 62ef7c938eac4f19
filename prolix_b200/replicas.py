"""Replica parallelism across GPUs: one process per GPU, each with its own
batch of independent systems, no collective on the data path.

The only cross-rank traffic is bookkeeping: a barrier around timed regions,
the maximum of the ranks' device times (the job is as slow as its slowest
rank) and the sum of their atom counts.  prolix's one multi-device hook,
``physics/sharding.py:245-316`` (pmap over the atom axis of one system with
a host-side sum), has no counterpart here: systems never span GPUs.
"""

from __future__ import annotations

import datetime
import os


def env():
  """(world_size, rank, local_rank) from the torchrun environment."""
  return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
          int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
  """Initialise the process group when launched with more than one rank."""
  import torch.distributed as dist
  ws, _, _ = env()
  if ws > 1 and not dist.is_initialized():
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
  return dist if ws > 1 else None


def rank_seed(base: int, rank: int) -> int:
  """Workload seed of a rank (each replica simulates different systems)."""
  return int(base) + 7919 * int(rank)


def _tensor(v, device):
  import torch
  return torch.tensor([float(v)], dtype=torch.float64, device=device)


def reduce_max(value: float, device="cpu") -> float:
  import torch.distributed as dist
  if not (dist.is_available() and dist.is_initialized()):
    return float(value)
  t = _tensor(value, device)
  dist.all_reduce(t, op=dist.ReduceOp.MAX)
  return float(t.item())


def reduce_sum(value: float, device="cpu") -> float:
  import torch.distributed as dist
  if not (dist.is_available() and dist.is_initialized()):
    return float(value)
  t = _tensor(value, device)
  dist.all_reduce(t, op=dist.ReduceOp.SUM)
  return float(t.item())


def barrier():
  import torch.distributed as dist
  if dist.is_available() and dist.is_initialized():
    dist.barrier()


def aggregate(local_ms: float, local_atoms: int, steps: int, device="cpu") -> dict:
  """Whole-job throughput of weakly scaled replicas: total atoms x steps over
  the slowest rank's time."""
  t = reduce_max(local_ms, device)
  atoms = reduce_sum(local_atoms, device)
  return {"ms": t, "atoms": int(atoms), "atom_steps_per_s": atoms * steps / (t * 1e-3)}
