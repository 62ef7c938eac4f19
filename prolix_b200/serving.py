"""Continuous-batching server for "run K Langevin steps of system S" jobs.

Requests that arrive while others run join the device batch at the next
tick: each tick advances every running system by the same number of steps
(at most ``chunk``, and never past the nearest completion), then finished,
cancelled or failed requests end, and waiting requests are admitted while
the running systems stay inside the atom and HBM budgets.  All systems of a
tick share one launch per kernel (the ragged batch), so short and long,
small and large jobs overlap on the GPU.  The batch is rebuilt when
requests are admitted (their initial momenta and forces come from one
langevin_init of the new batch) or when ended systems, which keep stepping
unread until then, hold a quarter of its atoms.

Systems never interact and forces use order-independent fixed-point sums,
so a request's result is bit-identical whether it ran alone or in any mix
(checked by tests/test_gpu_serving.py).  A request whose state turns
non-finite is evicted with an error; the others carry on unchanged.

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
  x: np.ndarray
  p: np.ndarray
  f: np.ndarray   # forces at x: a rebuilt batch restores them instead of re-evaluating
  key: np.ndarray
  done: int
  admitted: float


_FIELDS = ("position", "momentum", "force", "key")


def _percentile(v, q):
  return float(np.percentile(np.asarray(v), q)) if len(v) else float("nan")


class Server:
  """Admission by budget, resident state, continuous batching."""

  def __init__(self, device: int = 0, hbm_budget_bytes: float = 150e9,
               max_batch_atoms: int = 1_000_000, chunk: int = 50, cutoff: float = 0.0,
               clock=time.perf_counter, batch_factory=None):
    self.device = device
    self.batch_factory = batch_factory or engine.Batch
    self.hbm_budget = float(hbm_budget_bytes)
    self.max_atoms = int(max_batch_atoms)
    self.chunk = int(chunk)
    self.cutoff = float(cutoff)
    self.clock = clock
    self.t0 = clock()
    self.queue: deque[Request] = deque()
    self.active: list[_Slot] = []
    self.results: dict[int, Result] = {}
    self.cancelled: set[int] = set()
    self._next_id = 0
    self._batch = None
    self._slot_of: list = []  # batch system index -> running slot, None once its request ended
    self.atom_steps = 0
    self.ticks = 0
    if self.batch_factory is engine.Batch:
      engine.Context.get(device)  # open the device now, not inside the first request

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
    if "excl_pairs" not in req.system:  # once per request, not on every batch rebuild
      pairs, kind = topology.exclusion_pairs(req.system.get("bonds", np.zeros((0, 2))), n)
      req.system = dict(req.system, excl_pairs=pairs, excl_kind=kind)
    self.queue.append(req)
    return req.rid

  def cancel(self, rid: int):
    self.cancelled.add(rid)

  def idle(self) -> bool:
    return not self.queue and not self.active

  # ------------------------------------------------------------------ internals
  def _used(self):
    atoms = sum(len(s.req.system["charges"]) for s in self.active)
    return atoms, atoms * BYTES_PER_ATOM

  def _admit(self, now: float) -> list:
    """Take waiting requests while the budget allows (first come, first
    served); they join the batch at the next rebuild."""
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
      # fix the system's float32 frame for its lifetime (bit-identical forces
      # whatever batch it runs in)
      if req.system.get("origin") is None:
        req.system = dict(req.system, origin=engine.default_origin(req.system["positions"]))
      admitted.append(req)
      atoms += n
      used += n * BYTES_PER_ATOM
    return admitted

  def _fail(self, req, admitted, now, msg):
    self.results[req.rid] = Result(req.rid, None, None, None, 0, req.arrival, admitted, now,
                                   error=msg)

  def _build(self, admitted, now):
    """A new batch of the running systems and the admitted requests.  Each
    system is described by its submitted positions, which fix its stored
    atom order.  One langevin_init draws the admitted requests' momenta from
    their keys and evaluates their forces (the same bits as alone); then every
    running system's saved state is restored, forces included, since forces
    depend only on the system's own float32 frame."""
    run_sys = [dict(s.req.system, key=tuple(int(v) for v in s.key), dt=s.req.dt, kT=s.req.kT,
                    gamma=s.req.gamma) for s in self.active]
    new_sys = [dict(r.system, key=r.key, dt=r.dt, kT=r.kT, gamma=r.gamma) for r in admitted]
    if self._batch is not None:
      self._batch.close()
      self._batch = None
    batch = self.batch_factory(run_sys + new_sys, cutoff=self.cutoff, device=self.device,
                               graph_chunk=self.chunk)
    self._batch = batch
    nr = len(run_sys)
    slot_of = list(self.active)
    st = None
    if admitted:
      batch.langevin_init()
      st = batch.get_state(fields=_FIELDS)
      status = batch.status(clear=True)
      for k, r in enumerate(admitted):
        b = nr + k
        lo, hi = batch.offsets[b], batch.offsets[b + 1]
        x = st["position"][lo:hi]
        if status[b] & (STATUS_NONFINITE | STATUS_FORCE_RANGE) or not np.isfinite(x).all():
          self._fail(r, now, now, "non-finite initial state")
          slot_of.append(None)
          continue
        slot_of.append(_Slot(r, x.copy(), st["momentum"][lo:hi].copy(), st["force"][lo:hi].copy(),
                             st["key"][b].copy(), 0, now))
    self._slot_of = slot_of  # batch system index -> running slot (None: its request ended)
    self.active = [s for s in slot_of if s is not None]
    if nr:
      # the running systems' saved state (the admitted ones keep the init's)
      def rows(field, st_field):
        return np.concatenate([getattr(slot_of[b], field) if b < nr
                               else st[st_field][batch.offsets[b]:batch.offsets[b + 1]]
                               for b in range(len(slot_of))])
      keys = np.stack([slot_of[b].key if b < nr else st["key"][b] for b in range(len(slot_of))])
      batch.set_full_state(rows("x", "position"), rows("p", "momentum"), rows("f", "force"), key=keys)

  def _save(self):
    st = self._batch.get_state(fields=_FIELDS)
    for b, s in enumerate(self._slot_of):
      if s is None:
        continue
      lo, hi = self._batch.offsets[b], self._batch.offsets[b + 1]
      s.x = st["position"][lo:hi].copy()
      s.p = st["momentum"][lo:hi].copy()
      s.f = st["force"][lo:hi].copy()
      s.key = st["key"][b].copy()
    return self._batch.status(clear=True)

  def _ended_atoms(self) -> int:
    return sum(self._batch.sizes[b] for b, s in enumerate(self._slot_of) if s is None)

  def tick(self) -> bool:
    """Admit, advance every running system, retire.  False when idle.

    The batch is rebuilt only when requests are admitted, or when systems
    whose requests have ended make up more than a quarter of its atoms:
    until then they keep stepping unread (each system is independent, so
    the others' results do not change)."""
    now = self.now()
    admitted = self._admit(now)
    if self.cancelled:
      for b, s in enumerate(self._slot_of):
        if s is not None and s.req.rid in self.cancelled:
          self._slot_of[b] = None
      for s in self.active:
        if s.req.rid in self.cancelled and s.req.rid not in self.results:
          self._fail(s.req, s.admitted, now, "cancelled")
      self.active = [s for s in self.active if s.req.rid not in self.cancelled]
    if not self.active and not admitted:
      if self._batch is not None:
        self._batch.close()
        self._batch = None
        self._slot_of = []
      return bool(self.queue)
    if (admitted or self._batch is None
        or self._ended_atoms() * 4 > int(np.sum(self._batch.sizes))):
      self._build(admitted, now)
      if not self.active:
        return bool(self.queue)
    n = min(self.chunk, min(s.req.n_steps - s.done for s in self.active))
    self._batch.langevin_run(n)
    status = self._save()
    self.ticks += 1
    now = self.now()
    for b, s in enumerate(self._slot_of):
      if s is None:
        continue
      s.done += n
      self.atom_steps += n * len(s.req.system["charges"])
      ended = True
      if status[b] & (STATUS_NONFINITE | STATUS_FORCE_RANGE) or not np.isfinite(s.x).all():
        self._fail(s.req, s.admitted, now, "non-finite state: evicted")
      elif s.done >= s.req.n_steps:
        self.results[s.req.rid] = Result(s.req.rid, s.x, s.p, s.key, s.done, s.req.arrival,
                                         s.admitted, now)
      else:
        ended = False
      if ended:
        self._slot_of[b] = None
    self.active = [s for s in self._slot_of if s is not None]
    return True

  def run(self, requests=(), until_idle=True, sleep=time.sleep):
    """Feed requests at their arrival times (server clock) and serve them."""
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    while True:
      now = self.now()
      while pending and pending[0].arrival <= now:
        self.submit(pending.popleft())
      if self.active or (self.queue and self.queue[0].arrival <= now):
        self.tick()
      elif pending:
        sleep(max(0.0, pending[0].arrival - self.now()))
      elif self.queue:
        sleep(max(0.0, self.queue[0].arrival - self.now()))
      elif until_idle:
        break
    if self._batch is not None:
      self._batch.close()
      self._batch = None
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
            "ticks": self.ticks}


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
