#!/usr/bin/env python3
"""Benchmark: aggregate atom-steps/s of the batched implicit-solvent
Langevin step (ragged batch of seeded synthetic chains, all pairs), with the
plain one-batch-per-system path, end-to-end C-ABI throughput, a served
request stream (p50/p99 latency), the roofline of the dominant kernel and a
CPU baseline beside it.

One "step" = one BAOAB step (force evaluation included) of every system of
the batch.  Workload: 512 systems with atom counts log-uniform in
150-4,000 (seed 2024), OBC2 GB + Coulomb + LJ + bonded terms, all pairs,
dt = 1 fs, gamma = 1/ps, T = 300 K.  Charges and LJ parameters come from
synth.PHYSICAL_RANGES (|q| <= 0.5 e, sigma 2.4-3.4 A): with the generator's
wider default ranges nearly every system blows up within 100 steps, and the
pair kernels would then be timed on exploded geometry.

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
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

METRIC = "aggregate atom-steps/s (ragged batch, all pairs)"
UNIT = "atom-steps/s"
WORKLOAD_SEED = 2024
N_SYSTEMS = 512

# Algorithmic work per unique pair (i < j), counted from the kernel source
# with FMA = 2 flops (pb2_pair.cu bc_series2 / run_force_tile2).  The
# descreening and chain passes evaluate the far-field series V (value) or D
# (derivative) as a polynomial of K terms, K chosen per tile from the
# bounding-box separation (pb2_obc_series.cuh tiers: V 3-6 terms, D 4-7);
# series_terms() gives the pair-weighted mean K of each.
#   descreening: 3 (d) + 5 (r^2) + 2 (1/r^2, 1/r^4)
#                + 2 x (1 + 2(K-1) + 1) (u, polynomial, s^3) + 2 x 2 (sums) = 4K + 14
#   force:       8 (d, r^2) + GB 15 (w, f^2, 1/f^3, A2, g) + 4 (dE/dB)
#                + 1 (1/r^2) + Coulomb 2 + LJ 11 + 2 (sum) + 12 (F)      = 55
#   chain:       3 (d) + 5 (r^2) + 3 (1/r^2, -1/r^6)
#                + 2 x (1 + 2(K-1) + 1) + 4 (g) + 12 (F)                  = 4K + 27
def flops_per_pair(k_mean: dict) -> dict:
  return {"born": 4.0 * k_mean["value"] + 14.0, "force": 55.0, "chain": 4.0 * k_mean["deriv"] + 27.0}


def series_tiers() -> dict:
  """u bounds and term counts of the polynomial tiers the kernels use."""
  import re
  with open(os.path.join(ROOT, "prolix_b200", "csrc", "pb2_obc_series.cuh")) as f:
    txt = f.read()
  out = {}
  for name in ("Value", "Deriv"):
    u = re.search(r"k%sTierU\[4\] = \{([^}]*)\}" % name, txt).group(1)
    k = re.search(r"k%sTierTerms\[4\] = \{([^}]*)\}" % name, txt).group(1)
    out[name.lower()] = ([float(v) for v in u.split(",")], [int(v) for v in k.split(",")])
  return out


def series_terms(systems) -> dict:
  """Pair-weighted mean number of polynomial terms per tile (value and
  derivative series), by the same bounding-box classification the kernels
  use (float32 radii)."""
  tiers = series_tiers()
  tot = {"value": 0.0, "deriv": 0.0}
  tot_w = 0.0
  for sd in systems:
    x = np.asarray(sd["positions"], dtype=np.float64)
    n = len(x)
    sr = np.asarray(sd["scaled_radii"], dtype=np.float32).astype(np.float64)
    ro = (np.asarray(sd["radii"], dtype=np.float64) - 0.09).astype(np.float32).astype(np.float64)
    smax, romax = sr.max(), ro.max()
    b2 = lambda u: (1.001 * max(smax / math.sqrt(u), smax + romax)) ** 2
    nb = (n + 31) // 32
    m = np.minimum(32, n - 32 * np.arange(nb))
    lo = np.array([x[32 * b:32 * b + 32].min(0) for b in range(nb)])
    hi = np.array([x[32 * b:32 * b + 32].max(0) for b in range(nb)])
    ib, jb = np.triu_indices(nb)
    d = np.maximum(0.0, np.maximum(lo[ib] - hi[jb], lo[jb] - hi[ib]))
    d2 = (d * d).sum(1)
    w = np.where(ib == jb, m[ib] * (m[ib] - 1) / 2.0, m[ib] * m[jb].astype(np.float64))
    for key, (us, ks) in tiers.items():
      k = np.select([d2 >= b2(us[0]), d2 >= b2(us[1]), d2 >= b2(us[2])], [float(v) for v in ks[:3]],
                    float(ks[3]))
      tot[key] += float((k * w).sum())
    tot_w += float(w.sum())
  return {key: v / tot_w for key, v in tot.items()}


MUFU_PER_PAIR = {"born": 1, "force": 3, "chain": 1}
# The same passes counted with the closed-form OBC formulas that prolix
# evaluates for every pair (generalized_born.py:211-263 per ordered pair:
# about 40 flops for I_ij, 45 for dI_ij/dr; analytical_forces.py:167-292
# for GB + Coulomb + LJ: about 70 flops per unique pair), per unique pair.
# The series kernels do less arithmetic than this, so the equivalent rate
# can exceed the FP32 peak; it is reported beside the counted figure.
CLOSED_FORM_FLOPS_PER_PAIR = {"born": 80.0, "force": 70.0, "chain": 90.0}
# integrator: read x, p (48 B), F (24 B), mass, sigma, charge (24 B); write
# x, p (48 B), posq (16 B), clear F (24 B)
BYTES_PER_ATOM_STEP = 184
# DRAM traffic per launch of each pair pass on this workload
# (dram__bytes_read.sum + dram__bytes_write.sum of one `ncu --set full`
# capture of the three passes, default block shapes and fusion)
TRAFFIC_BYTES = {"born": 24.19e6, "force": 71.33e6, "chain": 127.59e6}


def parse():
  ap = argparse.ArgumentParser()
  ap.add_argument("--gpus", type=int, default=1)
  ap.add_argument("--steps", type=int, default=400)
  ap.add_argument("--warmup", type=int, default=3)
  ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
  ap.add_argument("--systems", type=int, default=N_SYSTEMS)
  ap.add_argument("--no-plain", action="store_true")
  ap.add_argument("--no-cpu", action="store_true")
  ap.add_argument("--no-e2e", action="store_true")
  ap.add_argument("--e2e-tune", type=int, default=1,
                  help="end-to-end leg: 1 runs the autotuner on the first group and applies its choice to all")
  ap.add_argument("--e2e-groups", type=lambda v: [int(x) for x in v.split(",")], default=[12],
                  help="streams the end-to-end leg splits the systems over (comma list; the first "
                       "is the reported value)")
  ap.add_argument("--clocks-dir", default=None,
                  help="folder for the nvidia-smi clock samples of the timed region "
                       "(default: a new folder under the system temporary folder)")
  ap.add_argument("--no-serving", action="store_true")
  ap.add_argument("--no-extra", action="store_true",
                  help="skip the single-system, neighbour-list and serving-sweep legs")
  ap.add_argument("--serving-requests", type=int, default=200,
                  help="requests per rate of the served stream")
  ap.add_argument("--serving-rates", type=lambda v: [float(x) for x in v.split(",")],
                  default=[10.0, 20.0, 50.0, 100.0, 200.0, 500.0],
                  help="arrival rates (req/s) of the serving sweep; the headline serving entry is "
                       "the 20 req/s one when present, else the first")
  ap.add_argument("--serving-step-scale", type=float, default=1.0,
                  help="scales the requests' step counts (1.0: log-uniform 1,000-50,000)")
  ap.add_argument("--keep-atom-order", action="store_true",
                  help="store atoms in input order instead of the default spatial order")
  ap.add_argument("--nlist-only", action="store_true",
                  help="only build the neighbour list of the 20,000-atom globule at 20 + 2 A "
                       "a few times (a short command for profiling the list build)")
  ap.add_argument("--segment", type=int, default=0,
                  help="tile work-item segment; 0 runs the autotuner")
  return ap.parse_args()


def dist_env():
  ws = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  return ws, rank, local


def workload(rank: int, n_systems: int):
  from prolix_b200 import replicas, synth
  return synth.make_batch(n_systems, replicas.rank_seed(WORKLOAD_SEED, rank), 150, 4000, compact=True,
                          **synth.PHYSICAL_RANGES)


def unique_pairs(systems) -> int:
  return int(sum(len(s["charges"]) * (len(s["charges"]) - 1) // 2 for s in systems))


def cpu_model():
  try:
    for line in open("/proc/cpuinfo"):
      if line.startswith("model name"):
        return line.split(":", 1)[1].strip()
  except OSError:
    pass
  return "unknown"


def cpu_reference_run(systems, budget_s=12.0, start=0):
  """The FP64 C/OpenMP restatement of prolix's force field (oracle/) on the
  host's cores: one force evaluation per system (the O(N) integrator update,
  under 0.1 % of a step, is left out, which favours the CPU), systems in
  workload order from ``start`` (wrapping) until the budget is spent or every
  system ran once.  Returns (atom-steps/s, sample, threads, next start)."""
  from oracle import cforces
  threads = cforces.threads()
  atoms, t_total, used = 0, 0.0, 0
  n = len(systems)
  while used < n:
    s = systems[(start + used) % n]
    t0 = time.perf_counter()
    cforces.energy_forces(s, threads=threads)
    t_total += time.perf_counter() - t0
    atoms += len(s["charges"])
    used += 1
    if t_total > budget_s:
      break
  sample = (f"{used} of {n} systems x 1 step ({atoms} atom-steps); FP64 C/OpenMP "
            "restatement of prolix's formulas (the reference's JAX path cannot run here: JAX "
            "is not installed)")
  return atoms / t_total, sample, threads, (start + used) % n


def cpu_numpy_run(systems, budget_s=10.0):
  """The FP64 NumPy restatement (oracle/energy.py, vectorised over pairs;
  NumPy's elementwise arithmetic runs on one thread): one force evaluation
  per system, in workload order, until the budget is spent.  Returns
  (atom-steps/s, sample)."""
  from oracle import energy
  atoms, t_total, used = 0, 0.0, 0
  for s in systems:
    t0 = time.perf_counter()
    energy.energy_forces(s, s["positions"])
    t_total += time.perf_counter() - t0
    atoms += len(s["charges"])
    used += 1
    if t_total > budget_s:
      break
  return atoms / t_total, (f"first {used} of {len(systems)} systems x 1 step ({atoms} atom-steps); "
                           "FP64 NumPy restatement of prolix's formulas")


def clocks_start(path):
  try:
    return subprocess.Popen(
        ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
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
  # about two minutes of CPU work in total; successive steps continue through
  # the workload where the previous one stopped, so the steps together sample
  # every system size in proportion
  budget = max(0.2, 120.0 / max(args.steps, 1))
  for _ in range(args.warmup):
    cpu_reference_run(systems[:1], budget_s=0.0)
  t0 = time.perf_counter()
  atoms_total, time_total, nxt = 0.0, 0.0, 0
  sample, threads = "", 1
  for _ in range(args.steps):
    v, sample, threads, start = cpu_reference_run(systems, budget_s=budget, start=nxt)
    n_used = (start - nxt) % len(systems) or len(systems)
    atoms = sum(len(systems[(nxt + k) % len(systems)]["charges"]) for k in range(n_used))
    atoms_total += atoms
    time_total += atoms / v
    nxt = start
  value = atoms_total / time_total
  sample = (f"{args.steps} steps of at most {budget:.2f} s each ({time_total / max(args.steps, 1):.2f} s on "
            f"average), continuing through the {len(systems)}-system workload ({int(atoms_total)} "
            f"atom-steps in all); " + sample.split("; ", 1)[1])
  line = {
      "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
      "steps": args.steps, "warmup": args.warmup,
      "ms_per_step": 1e3 * sum(len(s["charges"]) for s in systems) / value,
      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
      "data": "synthetic (seeded chains)",
      "config": {"workload": f"{args.systems} systems, N log-uniform 150-4000 (seed {WORKLOAD_SEED}), "
                             "OBC2 GB + Coulomb + LJ + bonded, all pairs, BAOAB dt 1 fs",
                 "parameters": "charges U(-0.5, 0.5) e, LJ sigma U(2.4, 3.4) A, eps U(0.03, 0.2)",
                 "parallelism": f"{threads} host threads"},
      "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                       "sample": sample, "cpu": cpu_model()},
      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
      "wall_s": time.perf_counter() - t0,
  }
  print(json.dumps(line), flush=True)
  return 0


def serving_sweep(args):
  """The served request stream at each rate: Poisson arrivals, N
  log-uniform 100-10,000 atoms, K log-uniform 1,000-50,000 steps (times
  --serving-step-scale), the same seeded requests at every rate, admitted
  against a 150 GB HBM budget into device-resident cohorts.  p50/p99 are
  end-to-end latencies (arrival to result on the host)."""
  from prolix_b200 import serving
  res = {}
  for rate in args.serving_rates:
    reqs = serving.poisson_requests(args.serving_requests, rate, WORKLOAD_SEED,
                                    step_scale=args.serving_step_scale)
    srv = serving.Server(chunk=50, hbm_budget_bytes=150e9)
    t0 = time.perf_counter()
    srv.run(reqs)
    rep = srv.report()
    rep["wall_s"] = time.perf_counter() - t0
    rep.update({"rate_per_s": rate, "atoms": "log-uniform 100-10,000",
                "steps": f"log-uniform 1,000-50,000 x {args.serving_step_scale}",
                "hbm_budget_gb": 150})
    res[str(int(rate))] = rep
  return res


def plain_run(systems, stream, steps):
  """The same systems with one batch (and one set of launches) per system."""
  import torch
  from prolix_b200 import engine
  batches = [engine.Batch([s]) for s in systems]
  for b in batches:
    b.langevin_init()
    for _ in range(2):  # one-step graphs of both key parities, captured before timing
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


def single_system_runs(stream, hbm_peak):
  """The single-system configurations.

  * config 1: the 166-atom chain, all pairs, 1,000 BAOAB steps at 1 fs;
  * config 2: N = 2,500 with CMAP and a 20 A cutoff, 2 A skin: the pair
    kernels step from the block-pair list rebuilt on the device on the
    half-skin rule, timed against the same run scanning every block pair
    (``pair_list=False``);
  * config 4: the 20,000-atom globule all pairs, and at 20 A (both ways).

  Device atom-steps/s of 50-step graph chunks.  For each cutoff run, the
  jax_md-layout neighbour list is built on the device: its device time
  (CUDA events around the build's launches, the median of 10 builds) and
  the bytes its rows write (every slot of every row) against the measured
  HBM bandwidth."""
  import torch
  from prolix_b200 import engine, synth

  def timed(b, steps):
    b.langevin_init()
    b.langevin_run(50, stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    b.langevin_run(steps, stream)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)

  out = {}
  for name, n, cutoff, steps, seed, cmap in (
      ("n166_all", 166, 0.0, 1000, 1, False), ("n2500_cut20", 2500, 20.0, 200, 2500, True),
      ("n20000_all", 20000, 0.0, 50, 4242, True), ("n20000_cut20", 20000, 20.0, 50, 4242, True)):
    sd = synth.make_chain(n, seed, compact=n > 166, cmap=cmap, **synth.PHYSICAL_RANGES)
    with engine.Batch([sd], cutoff=cutoff, skin=2.0) as b:
      ms = timed(b, steps)
      rec = {"atoms": n, "cutoff": cutoff, "steps": steps, "ms_per_step": ms / steps,
             "atom_steps_per_s": n * steps / (ms * 1e-3)}
      if cutoff > 0:
        rec["pair_list"] = "block pairs within cutoff + 2 A skin, rebuilt on the device at skin/2"
        b.nl_build(stream)  # sizes the rows
        cap = b.nl_capacity()
        times = []
        for _ in range(10):
          b.nl_build(stream)
          times.append(b.nl_last_build_ms())
        t = float(np.median(times)) * 1e-3
        nbytes = n * cap * 4
        rec["nlist"] = {"capacity": cap, "build_ms": t * 1e3, "bytes_written": nbytes,
                        "achieved_gbs": nbytes / t / 1e9, "peak_gbs": hbm_peak,
                        "frac": nbytes / t / 1e9 / hbm_peak,
                        "note": "device time of the cell-list build's launches (CUDA events), "
                                "median of 10; bytes = every slot of every row"}
    if cutoff > 0:
      with engine.Batch([sd], cutoff=cutoff, skin=2.0, pair_list=False) as b:
        ms2 = timed(b, steps)
      rec["without_pair_list"] = {"ms_per_step": ms2 / steps,
                                  "atom_steps_per_s": n * steps / (ms2 * 1e-3)}
    out[name] = rec
  return out


def split_run(systems, stream, born_cutoff=10.0, steps=100):
  """The NL-Born + dense-GB option on the timing batch: descreening and its
  chain rule within ``born_cutoff``, GB pair terms, Coulomb and LJ over all
  pairs.  Device atom-steps/s (no L2 flush; 50-step graphs)."""
  import torch
  from prolix_b200 import engine
  with engine.Batch(systems, born_cutoff=born_cutoff) as b:
    b.langevin_init()
    b.langevin_run(50, stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    b.langevin_run(steps, stream)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n = b.n_atoms
  return {"born_cutoff": born_cutoff, "ms_per_step": ms / steps,
          "atom_steps_per_s": n * steps / (ms * 1e-3)}


def minimize_run(systems, stream):
  """Throughput of the batched minimiser on the timing batch: 100 restrained
  steepest-descent steps and 4 FIRE stages of 50 iterations (the
  batched_minimize schedule, shortened), device time of the whole call."""
  import torch
  from prolix_b200 import engine, minimize
  with engine.Batch(systems) as b:
    b.min_setup()
    rms0 = b.min_rms()
    b.min_sd(5, k=minimize.SD_K, kind="heavy", dt=minimize.SD_DT, max_dx=minimize.SD_MAX_DX)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    b.min_sd(100, k=minimize.SD_K, kind="heavy", dt=minimize.SD_DT, max_dx=minimize.SD_MAX_DX)
    for k, kind in zip(minimize.FIRE_K, minimize.FIRE_KIND):
      b.min_fire(50, k=k, kind=kind, dt_start=minimize.FIRE_DT_START, dt_max=minimize.FIRE_DT_MAX,
                 max_disp=minimize.FIRE_MAX_DISP)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rms1 = b.min_rms()
    n = b.n_atoms
  iters = 100 + 4 * 50
  return {"iterations": iters, "ms": ms, "atom_iterations_per_s": n * iters / (ms * 1e-3),
          "rms_grad_median_before": float(np.median(rms0)), "rms_grad_median_after": float(np.median(rms1))}


def nlist_only():
  """Three device-side builds of the jax_md-layout list of the 20,000-atom
  globule (cutoff 20 A, skin 2 A), each timed with CUDA events."""
  from prolix_b200 import engine, synth
  sd = synth.make_chain(20000, 4242, compact=True, cmap=True, **synth.PHYSICAL_RANGES)
  with engine.Batch([sd], cutoff=20.0, skin=2.0) as b:
    b.nl_build()
    times = []
    for _ in range(3):
      b.nl_build()
      times.append(b.nl_last_build_ms())
    print(json.dumps({"nlist_build_ms": times, "capacity": b.nl_capacity()}))


def main():
  args = parse()
  if args.impl == "reference":
    return run_reference(args)
  if args.nlist_only:
    return nlist_only()
  import torch
  from prolix_b200 import replicas
  ws, rank, local = replicas.env()
  torch.cuda.set_device(local)
  pg = replicas.init("nccl", timeout_s=120.0)

  from prolix_b200 import engine
  systems = workload(rank, args.systems)
  n_atoms = int(sum(len(s["charges"]) for s in systems))
  # each rank has its own seeded systems: the job's atoms are their sum
  job_atoms = int(round(replicas.reduce_sum(float(n_atoms), device="cuda")))
  pairs = unique_pairs(systems)
  batch = engine.Batch(systems, device=local, keep_atom_order=args.keep_atom_order)
  batch.langevin_init()
  stream = torch.cuda.current_stream().cuda_stream

  from prolix_b200 import autotune
  if args.segment > 0:
    batch.set_tile_segment(args.segment)
    tuned = {"segment": args.segment, "timings": None}  # block shapes and fusion: defaults
  else:
    tuned = autotune.tune(batch, candidates=(2, 4, 8, 16, 32), steps=3, use_cache=False)
  batch_shapes = [batch.block_shape(p) for p in range(4)]
  batch_force_blocks = batch.force_blocks()
  batch_fusion = batch.fusion()
  for _ in range(args.warmup):  # also captures the one-step graph
    batch.langevin_run(1, stream)
  torch.cuda.synchronize()

  flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
  ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
  # a folder of this run's own unless one is given, so concurrent runs on a
  # host never share a sample file
  clk_dir = args.clocks_dir or tempfile.mkdtemp(prefix="pb2_clocks_")
  clk_path = os.path.join(clk_dir, f"clocks_rank{rank}_{os.getpid()}.csv")
  os.makedirs(os.path.dirname(clk_path), exist_ok=True)
  clk = clocks_start(clk_path)
  replicas.barrier()
  torch.cuda.synchronize()
  for k in range(args.steps):
    flush.zero_()  # evict L2 (256 MB > 126 MB) between timed steps
    ev0[k].record()
    batch.langevin_run(1, stream)
    ev1[k].record()
  torch.cuda.synchronize()
  replicas.barrier()
  clocks = clocks_summary(clk, clk_path, local)
  t_ms = replicas.reduce_max(float(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))), device="cuda")
  status = batch.status()
  if np.any(status):
    print(f"rank {rank}: status flags {np.unique(status)}", file=sys.stderr)
  value = job_atoms * args.steps / (t_ms * 1e-3)

  # per-kernel device times: eager launches with CUDA events around each
  batch.set_profiling(True)
  prof_steps = 5
  batch.langevin_run(prof_steps, stream)
  tim = batch.last_timings() / prof_steps  # ms per step
  batch.set_profiling(False)
  names = ["born", "finalize", "force", "chain", "bonded", "integrator", "bbox"]
  per_kernel = {n: float(v) for n, v in zip(names, tim[:7])}

  peak = ctypes_fp32_peak(batch)
  # XU (MUFU) peak: 16 lanes per SM per clock at the SM clock seen under load
  sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
  xu_peak = 16 * torch.cuda.get_device_properties(local).multi_processor_count * sm_mhz * 1e6 / 1e12
  passes = {}
  k_mean = series_terms(systems)
  fpp = flops_per_pair(k_mean)
  for p in ("born", "force", "chain"):
    ms = per_kernel[p]
    tf = fpp[p] * pairs / (ms * 1e-3) / 1e12 if ms > 0 else None
    mufu = MUFU_PER_PAIR[p] * pairs / (ms * 1e-3) / 1e12 if ms > 0 else None
    passes[p] = {"ms": ms, "tflops": tf, "frac": (tf / peak if tf and peak else None),
                 "mufu_tops": mufu, "xu_frac": mufu / xu_peak if mufu else None}
  dom = max(("born", "force", "chain"), key=lambda p: per_kernel[p])
  nominal = 128 * 2 * torch.cuda.get_device_properties(local).multi_processor_count * 1965e6 / 1e12
  roofline = {"kernel": f"tile_kernel pass '{dom}'", "bound": "fp32",
              "achieved": passes[dom]["tflops"], "peak": peak, "unit": "TFLOP/s",
              "frac": passes[dom]["frac"],
              "frac_of_nominal": (passes[dom]["tflops"] / nominal if passes[dom]["tflops"] else None),
              "nominal_peak": nominal,
              "traffic": TRAFFIC_BYTES.get(dom),
              "peak_source": "FP32 FMA throughput measured in this run (pb2_fp32_peak)",
              "xu_peak_tops": xu_peak,
              "algorithmic_flops_per_launch": fpp[dom] * pairs,
              "flops_per_pair": fpp, "series_terms_mean": k_mean,
              "passes": passes,
              "closed_form_equivalent": {
                  "flops_per_pair": CLOSED_FORM_FLOPS_PER_PAIR,
                  "tflops": {p: CLOSED_FORM_FLOPS_PER_PAIR[p] * pairs / (per_kernel[p] * 1e-3) / 1e12
                             for p in passes if per_kernel[p] > 0},
                  "frac": {p: CLOSED_FORM_FLOPS_PER_PAIR[p] * pairs / (per_kernel[p] * 1e-3) / 1e12 / peak
                           for p in passes if per_kernel[p] > 0 and peak}}}
  integ_gbs = BYTES_PER_ATOM_STEP * n_atoms / (per_kernel["integrator"] * 1e-3) / 1e9
  hbm_peak = _measured_hbm()
  integrator = {"achieved_gbs": integ_gbs, "peak_gbs": hbm_peak,
                "frac": integ_gbs / hbm_peak if hbm_peak else None,
                "bytes_per_atom_step": BYTES_PER_ATOM_STEP}

  e2e = None
  pipelined = None
  if not args.no_e2e:
    # every step: positions, momenta and forces in from page-locked host
    # buffers, one BAOAB step, and the same three arrays back out, through
    # pb2_langevin_run_host; the systems are split into groups of
    # consecutive systems, each a batch on its own stream, so that one
    # group's copies overlap another's steps (prolix_b200.streamed).  Timed
    # on the host clock around the calls, which return once every group's
    # state is back in host memory.
    from prolix_b200 import streamed
    e2e_steps = 10
    nbytes = 3 * 3 * 8 * n_atoms
    by_groups = {}
    group_choice = None
    for g in args.e2e_groups:
      with streamed.StreamedEnsemble(systems, groups=g, device=local) as ens:
        ens.langevin_init()
        if args.e2e_tune:
          # the groups are alike in size: the autotuner's choice for the first
          # serves them all (its timing steps advance that group's trajectory,
          # which the timed steps below then continue)
          choice = autotune.tune(ens.batches[0], candidates=(8, 16, 32), steps=3, use_cache=False)
          for bt in ens.batches:
            autotune.apply(bt, choice)
          if g == args.e2e_groups[0]:
            group_choice = choice
        host = ens.get_state()
        ens.synchronize()
        for it in range(2 + e2e_steps):
          if it == 2:
            torch.cuda.synchronize()
            replicas.barrier()
            t0 = time.perf_counter()
          ens.run_host(host["position"], host["momentum"], host["force"], 1)
        # every rank steps its own systems; the slowest rank's time counts
        t_e2e = replicas.reduce_max(time.perf_counter() - t0, device="cuda")
        by_groups[str(len(ens.batches))] = job_atoms * e2e_steps / t_e2e
        if g == args.e2e_groups[0]:
          # the same round trips queued without a host wait between steps
          # (each step still copies x, p, F in from and out to the host
          # arrays; the batches order each step's copy in after the previous
          # copy out), synchronised once at the end
          torch.cuda.synchronize()
          replicas.barrier()
          t0 = time.perf_counter()
          for _ in range(e2e_steps):
            ens.run_host(host["position"], host["momentum"], host["force"], 1, wait=False)
          ens.synchronize()
          t_pipe = replicas.reduce_max(time.perf_counter() - t0, device="cuda")
          pipelined = job_atoms * e2e_steps / t_pipe
    head = str(min(args.e2e_groups[0], len(systems)))
    e2e = {"value": by_groups[head], "unit": UNIT,
           "h2d_bytes_per_step": int(nbytes), "d2h_bytes_per_step": int(nbytes),
           "steps": e2e_steps, "host_buffers": "page-locked", "groups": int(head),
           "group_tuning": None if group_choice is None else
           {k: group_choice.get(k) for k in ("segment", "shapes", "force_blocks", "fusion")},
           "by_groups": by_groups,
           "pipelined_no_host_wait": pipelined,
           "path": "pb2_langevin_run_host(1 step, x, p, F) per group of systems, one stream per group; "
                   "the host waits for every step's state before the next (pipelined_no_host_wait: "
                   "the same round trips without that wait)"}
  batch.close()

  plain = None
  serving_rep = None
  cpu = None
  cpu_numpy = None
  if rank == 0:
    if not args.no_plain:
      plain = plain_run(systems, stream, steps=10)
    sweep = None
    if not args.no_serving:
      sweep = serving_sweep(args)
      head = "20" if "20" in sweep else next(iter(sweep))
      serving_rep = dict(sweep[head], sweep={k: {f: v[f] for f in (
          "completed", "failed", "p50_s", "p99_s", "atom_steps_per_s", "span_s", "wall_s",
          "cohorts", "ticks")} for k, v in sweep.items()})
    extra = None
    if not args.no_extra:
      extra = {"single_system": single_system_runs(stream, hbm_peak),
               "minimize": minimize_run(systems, stream),
               "nl_born_dense_gb": split_run(systems, stream)}
    if not args.no_cpu:
      v, sample, threads, _ = cpu_reference_run(systems, budget_s=12.0)
      cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
             "cpu": cpu_model()}
      vn, sample_n = cpu_numpy_run(systems, budget_s=10.0)
      cpu_numpy = {"value": vn, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample_n}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair (fixed-point sums) / f64 state",
        "data": "synthetic (seeded chains)",
        "config": {"workload": f"{args.systems} systems, N log-uniform 150-4000 (seed {WORKLOAD_SEED}), "
                               "OBC2 GB + Coulomb + LJ + bonded, all pairs, BAOAB dt 1 fs",
                   "parameters": "charges U(-0.5, 0.5) e, LJ sigma U(2.4, 3.4) A, eps U(0.03, 0.2)",
                   "atoms_per_gpu": n_atoms, "unique_pairs_per_gpu": pairs,
                   "parallelism": f"replicas x{ws}",
                   "l2": "256 MB buffer written between timed steps",
                   "tile_segment": tuned["segment"],
                   "block_shapes": {p: list(batch_shapes[k]) for k, p in
                                    enumerate(("born", "force", "chain", "force_four_blocks"))},
                   "force_iblocks_per_warp": batch_force_blocks,
                   "fusion": {"bonded_in_chain": bool(batch_fusion & 1),
                              "born_finalize_in_descreening": bool(batch_fusion & 2)},
                   "autotune_ms_per_step": tuned["timings"]},
        "clocks": clocks,
        "roofline": roofline,
        "integrator_roofline": integrator,
        "kernel_ms_per_step": per_kernel,
        "plain": plain,
        "ragged_over_plain": value / (plain["value"] * ws) if plain else None,
        "serving": serving_rep,
        "extra": extra,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "cpu_baseline_numpy": cpu_numpy,
        # per timed step (a one-step graph): the step kernel (with the block
        # boxes), the descreening, force and chain passes, the Born finalize
        # and the bonded terms unless fused into those passes, and the
        # closing half kick of the one-step run
        "gpu_launches": int(args.steps * (5 + (0 if batch_fusion & 1 else 1) + (0 if batch_fusion & 2 else 1))),
    }
    print(json.dumps(line), flush=True)
  if pg:
    pg.destroy_process_group()
  return 0


def ctypes_fp32_peak(batch):
  import ctypes
  v = ctypes.c_double(0.0)
  rc = batch.lib.pb2_fp32_peak(batch.ctx.handle, ctypes.byref(v))
  return v.value if rc == 0 else None


def _measured_hbm():
  try:
    return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
  except (OSError, KeyError, ValueError):
    return 6650.0  # the profiling recipe's fallback


if __name__ == "__main__":
  sys.exit(main())
