"""Continuous-batching server for "run K Langevin steps of system S" jobs.

Requests that arrive while others run are admitted at the next tick, while
the running systems stay inside the atom and HBM budgets.  Each admission
wave becomes a cohort: one device batch holding just the admitted systems,
created from their descriptions (the only upload) and initialised on the
device.  Running cohorts are never rebuilt and their state never leaves the
device: each tick advances every cohort by the same number of steps on its
own CUDA stream, so all cohorts' kernels overlap on the GPU, and only a
cohort in which a request has just finished is read back (the finished
systems' positions, momenta and keys are the result).  A system whose
request has ended is retired inside its cohort (stream-ordered; the pair
kernels' work list is compacted on the device), so it costs no more steps;
a cohort whose requests have all ended is released.

The step count of a tick is the largest of chunk, chunk/2, chunk/5,
chunk/10, 1 (and 1-step divisions thereof) that does not pass the nearest
completion, so every cohort captures at most a handful of step graphs.

Systems never interact and forces use order-independent fixed-point sums,
so a request's result is bit-identical whether it ran alone or in any mix
(checked by tests/test_gpu_serving.py).  A request whose state turns
non-finite (the step kernels' status bits) is evicted with an error; the
others carry on unchanged.

This has no counterpart in prolix (whose batched runs are offline
``batched_produce`` calls, batched_simulate.py:1125-1163); it drives the
same BAOAB step.
"""

from __future__ import annotations

import dataclasses
import math
import time
from collections import deque

import numpy as np

from . import engine, topology
from ._lib import STATUS_FORCE_RANGE, STATUS_NONFINITE

BYTES_PER_ATOM = 320  # device footprint of one atom in a batch (state, pair data, scratch)


@dataclasses.dataclass
class Request:
  system: dict
  n_steps: int
  key: tuple = (0, 0)
  dt: float = engine.akma_dt(1.0)
  kT: float = 300.0 * engine.KB_KCAL
  gamma: float = engine.akma_gamma(1.0)
  arrival: float = 0.0          # seconds (server clock)
  rid: int = -1


@dataclasses.dataclass
class Result:
  rid: int
  position: np.ndarray | None
  momentum: np.ndarray | None
  key: np.ndarray | None
  steps: int
  arrival: float
  admitted: float
  finished: float
  error: str | None = None

  @property
  def latency(self) -> float:
    return self.finished - self.arrival


@dataclasses.dataclass
class _Slot:
  req: Request
  done: int
  admitted: float


class _Cohort:
  """The systems admitted together: one device batch, one stream."""

  def __init__(self, batch, slots, stream):
    self.batch = batch
    self.slots = slots    # batch system index -> running slot, None once its request ended
    self.stream = stream  # a stream object with a .cuda_stream handle, or None

  def live(self) -> bool:
    return any(s is not None for s in self.slots)

  def end(self, b: int):
    """Request b's slot is over: retire its system (no further work)."""
    self.slots[b] = None
    if any(s is not None for s in self.slots):  # else the whole cohort is released
      self.batch.retire(b, self.stream.cuda_stream if self.stream is not None else None)

  def atoms(self) -> int:
    return int(np.sum(self.batch.sizes))


_FIELDS = ("position", "momentum", "key")


def _percentile(v, q):
  return float(np.percentile(np.asarray(v), q)) if len(v) else float("nan")


def _tick_steps(chunk: int, limit: int) -> int:
  """The largest of chunk, chunk/2, chunk/5, chunk/10 and 1 not above limit."""
  for d in (1, 2, 5, 10):
    n = max(1, chunk // d)
    if n <= limit:
      return n
  return 1


class Server:
  """Admission by budget, device-resident cohorts, continuous batching."""

  def __init__(self, device: int = 0, hbm_budget_bytes: float = 150e9,
               max_batch_atoms: int = 1_000_000, chunk: int = 50, cutoff: float = 0.0,
               clock=time.perf_counter, batch_factory=None, stream_factory=None):
    self.device = device
    self.batch_factory = batch_factory or engine.Batch
    self.hbm_budget = float(hbm_budget_bytes)
    self.max_atoms = int(max_batch_atoms)
    self.chunk = int(chunk)
    self.cutoff = float(cutoff)
    self.clock = clock
    self.t0 = clock()
    self.queue: deque[Request] = deque()
    self.cohorts: list[_Cohort] = []
    self.results: dict[int, Result] = {}
    self.cancelled: set[int] = set()
    self._next_id = 0
    self.atom_steps = 0
    self.ticks = 0
    self.cohorts_created = 0
    self.readbacks = 0
    self._streams = stream_factory
    self._sync = None
    if self.batch_factory is engine.Batch:
      engine.Context.get(device)  # open the device now, not inside the first request
      if self._streams is None:
        import torch
        self._streams = lambda: torch.cuda.Stream(device=device)
        self._sync = lambda: torch.cuda.synchronize(device)

  # ------------------------------------------------------------------ api
  def now(self) -> float:
    return self.clock() - self.t0

  def submit(self, req: Request) -> int:
    if req.rid < 0:
      req.rid = self._next_id
      self._next_id += 1
    else:
      self._next_id = max(self._next_id, req.rid + 1)
    n = len(req.system["charges"])
    if n * BYTES_PER_ATOM > self.hbm_budget or n > self.max_atoms:
      self.results[req.rid] = Result(req.rid, None, None, None, 0, req.arrival, float("nan"),
                                     self.now(), error="system larger than the server budget")
      return req.rid
    if "excl_pairs" not in req.system:  # once per request, not per cohort
      pairs, kind = topology.exclusion_pairs(req.system.get("bonds", np.zeros((0, 2))), n)
      req.system = dict(req.system, excl_pairs=pairs, excl_kind=kind)
    self.queue.append(req)
    return req.rid

  def cancel(self, rid: int):
    self.cancelled.add(rid)

  @property
  def active(self) -> list:
    """Running requests' slots."""
    return [s for c in self.cohorts for s in c.slots if s is not None]

  def idle(self) -> bool:
    return not self.queue and not self.cohorts

  # ------------------------------------------------------------------ internals
  def _used(self):
    atoms = sum(c.atoms() for c in self.cohorts)  # ended systems still hold their memory
    return atoms, atoms * BYTES_PER_ATOM

  def _admit(self, now: float) -> list:
    """Take waiting requests while the budget allows (first come, first served)."""
    atoms, used = self._used()
    admitted = []
    while self.queue and self.queue[0].arrival <= now:
      req = self.queue[0]
      if req.rid in self.cancelled:
        self.queue.popleft()
        self.results[req.rid] = Result(req.rid, None, None, None, 0, req.arrival, float("nan"),
                                       now, error="cancelled")
        continue
      n = len(req.system["charges"])
      if atoms + n > self.max_atoms or used + n * BYTES_PER_ATOM > self.hbm_budget:
        break  # first-come first-served: wait for room
      self.queue.popleft()
      admitted.append(req)
      atoms += n
      used += n * BYTES_PER_ATOM
    return admitted

  def _fail(self, req, admitted, now, msg):
    self.results[req.rid] = Result(req.rid, None, None, None, 0, req.arrival, admitted, now,
                                   error=msg)

  def _new_cohort(self, admitted, now):
    """A batch of just the admitted requests: their descriptions are the
    only upload; momenta and forces come from one langevin_init."""
    systems = [dict(r.system, key=r.key, dt=r.dt, kT=r.kT, gamma=r.gamma) for r in admitted]
    batch = self.batch_factory(systems, cutoff=self.cutoff, device=self.device,
                               graph_chunk=self.chunk)
    self.cohorts_created += 1
    batch.langevin_init()
    status = batch.status(clear=True)
    slots = []
    for k, r in enumerate(admitted):
      if status[k] & (STATUS_NONFINITE | STATUS_FORCE_RANGE):
        self._fail(r, now, now, "non-finite initial state")
        slots.append(None)
      else:
        slots.append(_Slot(r, 0, now))
    cohort = _Cohort(batch, slots, self._streams() if self._streams else None)
    for b, s in enumerate(slots):
      if s is None and cohort.live():
        batch.retire(b, cohort.stream.cuda_stream if cohort.stream is not None else None)
    if cohort.live():
      self.cohorts.append(cohort)
    else:
      batch.close()

  def _retire(self):
    keep = []
    for c in self.cohorts:
      if c.live():
        keep.append(c)
      else:
        c.batch.close()
    self.cohorts = keep

  def tick(self) -> bool:
    """Admit, advance every cohort, retire.  False when idle."""
    now = self.now()
    admitted = self._admit(now)
    if self.cancelled:
      for c in self.cohorts:
        for b, s in enumerate(c.slots):
          if s is not None and s.req.rid in self.cancelled:
            if s.req.rid not in self.results:
              self._fail(s.req, s.admitted, now, "cancelled")
            c.end(b)
    if admitted:
      self._new_cohort(admitted, now)
    self._retire()
    if not self.cohorts:
      return bool(self.queue)
    remaining = min(s.req.n_steps - s.done for s in self.active)
    n = _tick_steps(self.chunk, remaining)
    for c in self.cohorts:
      c.batch.langevin_run(n, c.stream.cuda_stream if c.stream is not None else None)
    if self._sync:
      self._sync()
    self.ticks += 1
    now = self.now()
    for c in self.cohorts:
      status = c.batch.status(clear=True)
      st = None
      for b, s in enumerate(c.slots):
        if s is None:
          continue
        s.done += n
        self.atom_steps += n * len(s.req.system["charges"])
        if status[b] & (STATUS_NONFINITE | STATUS_FORCE_RANGE):
          self._fail(s.req, s.admitted, now, "non-finite state: evicted")
          c.end(b)
        elif s.done >= s.req.n_steps:
          if st is None:  # a finished request: the cohort's state comes back once
            st = c.batch.get_state(fields=_FIELDS)
            self.readbacks += 1
          lo, hi = c.batch.offsets[b], c.batch.offsets[b + 1]
          x = st["position"][lo:hi].copy()
          if not np.isfinite(x).all():
            self._fail(s.req, s.admitted, now, "non-finite state: evicted")
          else:
            self.results[s.req.rid] = Result(s.req.rid, x, st["momentum"][lo:hi].copy(),
                                             st["key"][b].copy(), s.done, s.req.arrival,
                                             s.admitted, now)
          c.end(b)
    self._retire()
    return True

  def run(self, requests=(), until_idle=True, sleep=time.sleep):
    """Feed requests at their arrival times (server clock) and serve them."""
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    while True:
      now = self.now()
      while pending and pending[0].arrival <= now:
        self.submit(pending.popleft())
      if self.cohorts or (self.queue and self.queue[0].arrival <= now):
        self.tick()
      elif pending:
        sleep(max(0.0, pending[0].arrival - self.now()))
      elif self.queue:
        sleep(max(0.0, self.queue[0].arrival - self.now()))
      elif until_idle:
        break
    for c in self.cohorts:
      c.batch.close()
    self.cohorts = []
    return self.results

  def report(self) -> dict:
    ok = [r for r in self.results.values() if r.error is None]
    lat = [r.latency for r in ok]
    span = max((r.finished for r in ok), default=0.0) - min((r.arrival for r in ok), default=0.0)
    return {"requests": len(self.results), "completed": len(ok),
            "failed": len(self.results) - len(ok),
            "p50_s": _percentile(lat, 50), "p99_s": _percentile(lat, 99),
            "atom_steps": int(self.atom_steps), "span_s": span,
            "atom_steps_per_s": self.atom_steps / span if span > 0 else float("nan"),
            "ticks": self.ticks, "cohorts": self.cohorts_created, "readbacks": self.readbacks}


def poisson_requests(n: int, rate: float, seed: int, n_lo=100, n_hi=10_000, k_lo=1_000,
                     k_hi=50_000, step_scale=1.0, ranges=None):
  """Seeded request stream: Poisson arrivals at ``rate``/s, atoms and steps
  log-uniform; ``step_scale`` shrinks the step counts for bounded runs.
  Systems use ``synth.PHYSICAL_RANGES`` unless ``ranges`` is given."""
  from . import synth
  ranges = synth.PHYSICAL_RANGES if ranges is None else ranges
  rng = np.random.default_rng(seed)
  t = np.cumsum(rng.exponential(1.0 / rate, size=n))
  sizes = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), size=n)).astype(int)
  steps = np.exp(rng.uniform(math.log(k_lo), math.log(k_hi), size=n))
  steps = np.maximum(1, (steps * step_scale).astype(int))
  reqs = []
  for i in range(n):
    sys_ = synth.make_chain(int(sizes[i]), seed * 100003 + i, compact=True, **ranges)
    reqs.append(Request(system=sys_, n_steps=int(steps[i]), key=(0, int(seed * 7 + i)),
                        arrival=float(t[i]), rid=i))
  return reqs
