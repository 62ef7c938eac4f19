#!/usr/bin/env python3
"""Benchmark: aggregate atom-steps/s of the batched implicit-solvent
Langevin step (ragged batch of seeded synthetic chains, all pairs).

One "step" = one BAOAB step (force evaluation included) of every system of
the batch.  Workload: 512 systems with atom counts log-uniform in
150-4,000 (seed 2024), OBC2 GB + Coulomb + LJ + bonded terms, all pairs,
dt = 1 fs, gamma = 1/ps, T = 300 K.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank runs its own batch (replicas; seed offset by rank),
the timed region is bracketed by barriers and device syncs, and the slowest
rank's time defines the aggregate.  Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

METRIC = "aggregate atom-steps/s (ragged batch, all pairs)"
UNIT = "atom-steps/s"
WORKLOAD_SEED = 2024
N_SYSTEMS = 512


def parse():
  ap = argparse.ArgumentParser()
  ap.add_argument("--gpus", type=int, default=1)
  ap.add_argument("--steps", type=int, default=20)
  ap.add_argument("--warmup", type=int, default=3)
  ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
  ap.add_argument("--systems", type=int, default=N_SYSTEMS)
  ap.add_argument("--no-plain", action="store_true")
  ap.add_argument("--no-cpu", action="store_true")
  ap.add_argument("--no-e2e", action="store_true")
  return ap.parse_args()


def dist_env():
  ws = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  return ws, rank, local


def workload(rank: int, n_systems: int):
  from prolix_b200 import synth
  return synth.make_batch(n_systems, WORKLOAD_SEED + 7919 * rank, 150, 4000, compact=True)


def cpu_model():
  try:
    for line in open("/proc/cpuinfo"):
      if line.startswith("model name"):
        return line.split(":", 1)[1].strip()
  except OSError:
    pass
  return "unknown"


def cpu_reference_run(systems, budget_s=12.0, steps_per_sys=1):
  """Time the FP64 CPU restatement (oracle) on a bounded sample: one BAOAB
  step (one force evaluation) per system, systems taken in workload order
  until the budget is spent.  Returns (atom-steps/s, sample description)."""
  from oracle import energy as oenergy
  from oracle import integrator as ointeg
  from oracle import prng
  dt, kT, gamma = 1.0 / 48.88821291839, 300 * 0.0019872041, 48.88821291839e-3
  atoms = 0
  t_total = 0.0
  used = 0
  for s in systems:
    force = lambda r, s=s: oenergy.energy_forces(s, r)[1]
    st = ointeg.State(s["positions"], np.zeros_like(s["positions"]), np.zeros_like(s["positions"]),
                      s["masses"], prng.prng_key(1))
    t0 = time.perf_counter()
    ointeg.run(st, force, steps_per_sys, dt, kT, gamma)
    t_total += time.perf_counter() - t0
    atoms += len(s["charges"]) * steps_per_sys
    used += 1
    if t_total > budget_s:
      break
  return atoms / t_total, f"{used} of {len(systems)} systems x {steps_per_sys} step(s), {atoms} atom-steps"


def clocks_start(path):
  try:
    return subprocess.Popen(
        ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
        stdout=open(path, "w"), stderr=subprocess.DEVNULL)
  except OSError:
    return None


def clocks_summary(proc, path, device):
  if proc is None:
    return None
  proc.terminate()
  try:
    proc.wait(timeout=5)
  except subprocess.TimeoutExpired:
    proc.kill()
  sm, mx, reasons = [], None, set()
  names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
  try:
    for line in open(path):
      f = [x.strip() for x in line.split(",")]
      if len(f) < 9 or f[0] != str(device):
        continue
      try:
        sm.append(float(f[1]))
        mx = float(f[2])
      except ValueError:
        continue
      for n, v in zip(names, f[5:9]):
        if v.lower() == "active":
          reasons.add(n)
  except OSError:
    return None
  if not sm:
    return None
  return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
          "samples": len(sm)}


def run_reference(args):
  ws, rank, _ = dist_env()
  if rank != 0:
    return 0
  systems = workload(0, args.systems)
  per_step = []
  for _ in range(args.warmup):
    cpu_reference_run(systems[:1], budget_s=0.0)
  t0 = time.perf_counter()
  vals = []
  for _ in range(args.steps):
    v, sample = cpu_reference_run(systems, budget_s=max(2.0, 60.0 / max(args.steps, 1)))
    vals.append(v)
  el = time.perf_counter() - t0
  value = float(np.mean(vals))
  cores = 1
  line = {
      "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
      "steps": args.steps, "warmup": args.warmup,
      "ms_per_step": 1e3 * sum(int(s["charges"].shape[0]) for s in systems) / value,
      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
      "data": "synthetic (seeded chains)",
      "config": {"workload": f"{args.systems} systems, N log-uniform 150-4000, all pairs",
                 "parallelism": "host cores"},
      "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                       "sample": sample + "; FP64 NumPy restatement of prolix (the reference's "
                       "JAX path cannot run here: JAX is not installed)",
                       "cpu": cpu_model()},
      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
      "wall_s": el,
  }
  print(json.dumps(line), flush=True)
  return 0


def main():
  args = parse()
  if args.impl == "reference":
    return run_reference(args)
  import torch
  ws, rank, local = dist_env()
  torch.cuda.set_device(local)
  pg = None
  if ws > 1:
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pg = dist

  from prolix_b200 import engine
  systems = workload(rank, args.systems)
  n_atoms = int(sum(len(s["charges"]) for s in systems))
  batch = engine.Batch(systems, device=local)
  batch.langevin_init()
  stream = torch.cuda.current_stream().cuda_stream

  # warm-up (also captures the one-step graph)
  for _ in range(args.warmup):
    batch.langevin_run(1, stream)
  torch.cuda.synchronize()

  flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
  ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  clk_path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{rank}.csv")
  os.makedirs(os.path.dirname(clk_path), exist_ok=True)
  clk = clocks_start(clk_path)
  if pg:
    pg.barrier()
  torch.cuda.synchronize()
  for k in range(args.steps):
    flush.zero_()  # evict L2 (256 MB > 126 MB) between timed steps
    ev0[k].record()
    batch.langevin_run(1, stream)
    ev1[k].record()
  torch.cuda.synchronize()
  if pg:
    pg.barrier()
  clocks = clocks_summary(clk, clk_path, local)
  t_ms = float(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1)))
  if pg:
    t = torch.tensor([t_ms], device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    t_ms = float(t.item())
  status = batch.status()
  if np.any(status):
    print(f"rank {rank}: status flags {np.unique(status)}", file=sys.stderr)

  total_atoms = n_atoms * ws
  value = total_atoms * args.steps / (t_ms * 1e-3)

  # per-kernel device times (eager launches with events around each family)
  batch.set_profiling(True)
  prof_steps = max(3, min(args.steps, 10))
  batch.langevin_run(prof_steps, stream)
  tim = batch.last_timings() / prof_steps
  batch.set_profiling(False)

  # end to end through the C ABI with host buffers: upload state, one step,
  # read positions back, every step
  e2e = None
  if not args.no_e2e:
    st = batch.get_state()
    x_h, p_h = st["position"].copy(), st["momentum"].copy()
    e2e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
      batch.set_state(position=x_h, momentum=p_h)
      batch.langevin_run(1, stream)
      out = batch.get_state()
      x_h, p_h = out["position"], out["momentum"]
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    e2e = {"value": total_atoms * e2e_steps / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": int(2 * 3 * 8 * n_atoms),
           "d2h_bytes_per_step": int((3 * 3 * 8 + 3 * 8) * n_atoms),
           "steps": e2e_steps}

  plain = None
  if rank == 0 and not args.no_plain:
    plain = plain_run(systems, stream, steps=max(2, min(args.steps, 5)))

  if rank == 0:
    cpu = None
    if not args.no_cpu:
      v, sample = cpu_reference_run(systems, budget_s=12.0)
      cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
             "sample": sample + "; FP64 NumPy restatement of prolix (reference JAX path unavailable)",
             "cpu": cpu_model()}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair / f64 state",
        "data": "synthetic (seeded chains)",
        "config": {"workload": f"{args.systems} systems, N log-uniform 150-4000 (seed {WORKLOAD_SEED}), "
                               "OBC2 GB + Coulomb + LJ + bonded, all pairs, BAOAB dt 1 fs",
                   "atoms_per_gpu": n_atoms, "parallelism": f"replicas x{ws}",
                   "l2": "256 MB buffer written between timed steps"},
        "clocks": clocks,
        "kernel_ms_per_step": {"pair_and_bonded": tim[0], "integrator": tim[2]},
        "plain": plain,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "gpu_launches": int(args.steps * 6),
    }
    print(json.dumps(line), flush=True)
  batch.close()
  if pg:
    pg.destroy_process_group()
  return 0


def plain_run(systems, stream, steps):
  """The same systems with one batch (and one set of launches) per system."""
  import torch
  from prolix_b200 import engine
  batches = [engine.Batch([s]) for s in systems]
  for b in batches:
    b.langevin_init()
    b.langevin_run(1, stream)
  torch.cuda.synchronize()
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record()
  for _ in range(steps):
    for b in batches:
      b.langevin_run(1, stream)
  e1.record()
  torch.cuda.synchronize()
  ms = e0.elapsed_time(e1)
  n = sum(len(s["charges"]) for s in systems)
  for b in batches:
    b.close()
  return {"value": n * steps / (ms * 1e-3), "unit": UNIT, "steps": steps,
          "note": "one batch per system, launches issued system after system"}


if __name__ == "__main__":
  sys.exit(main())
