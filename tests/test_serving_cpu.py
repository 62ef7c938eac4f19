"""Scheduling logic of the continuous-batching server, on the CPU with a
stand-in batch that advances positions deterministically."""

import numpy as np

from prolix_b200 import serving


class FakeBatch:
  """x += 0.001 * steps per system; p counts steps; keys untouched."""

  def __init__(self, systems, **kw):
    self.sizes = [len(s["charges"]) for s in systems]
    self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
    self.x = np.concatenate([np.asarray(s["positions"], float) for s in systems])
    self.p = np.zeros_like(self.x)
    self.k = np.array([s["key"] for s in systems], dtype=np.uint32).reshape(-1, 2)
    self.n_systems = len(systems)
    self.retired = []

  def __enter__(self):
    return self

  def __exit__(self, *a):
    pass

  def close(self):
    pass

  def langevin_init(self):
    pass

  def langevin_run(self, n, stream=None):
    live = np.ones(len(self.x), bool)
    for s in self.retired:  # retired systems are not stepped
      live[self.offsets[s]:self.offsets[s + 1]] = False
    self.x = np.where(live[:, None], self.x + 0.001 * n, self.x)
    self.p = np.where(live[:, None], self.p + n, self.p)

  def retire(self, system, stream=None):
    assert system not in self.retired
    self.retired.append(system)

  def get_state(self, fields=("position", "momentum", "key")):
    st = {"position": self.x.copy(), "momentum": self.p.copy(), "key": self.k.copy(),
          "force": -self.x.copy()}
    return {f: st[f] for f in fields}

  def set_full_state(self, position, momentum, force, key=None):
    assert np.array_equal(force, -position)  # the forces saved with these positions
    self.set_state(position=position, momentum=momentum, key=key)

  def set_state(self, position=None, momentum=None, key=None):
    self.x, self.p, self.k = position.copy(), momentum.copy(), key.copy()

  def status(self, clear=False):
    bad = [not np.isfinite(self.x[self.offsets[s]:self.offsets[s + 1]]).all()
           for s in range(self.n_systems)]
    return np.array([1 if b else 0 for b in bad], dtype=np.uint32)


def _req(rid, n, steps, t):
  sys_ = {"charges": np.zeros(n), "positions": np.zeros((n, 3))}
  return serving.Request(system=sys_, n_steps=steps, key=(0, rid), arrival=t, rid=rid)


class Clock:
  def __init__(self):
    self.t = 0.0

  def __call__(self):
    return self.t

  def sleep(self, d):
    self.t += max(d, 1e-3)


def test_steps_exact_and_budget_respected():
  clk = Clock()
  srv = serving.Server(chunk=10, max_batch_atoms=100, clock=clk, batch_factory=FakeBatch)
  reqs = [_req(0, 60, 25, 0.0), _req(1, 50, 7, 0.0), _req(2, 30, 40, 0.5)]
  orig_tick = srv.tick
  seen = []

  def tick():
    seen.append(sum(len(s.req.system["charges"]) for s in srv.active))
    clk.t += 0.01
    return orig_tick()

  srv.tick = tick
  res = srv.run(reqs, sleep=clk.sleep)
  for r in reqs:
    assert res[r.rid].error is None
    assert res[r.rid].steps == r.n_steps
    np.testing.assert_allclose(res[r.rid].momentum, r.n_steps)  # exactly n_steps advanced
  assert max(seen) <= 100


def test_failure_is_isolated_and_reported():
  clk = Clock()
  srv = serving.Server(chunk=10, clock=clk, batch_factory=FakeBatch)
  bad = _req(1, 5, 20, 0.0)
  bad.system["positions"] = np.full((5, 3), np.nan)
  res = srv.run([_req(0, 5, 20, 0.0), bad], sleep=clk.sleep)
  assert res[1].error is not None and res[0].error is None


def test_poisson_stream_is_seeded():
  a = serving.poisson_requests(5, 50.0, 3, n_hi=300, step_scale=0.01)
  b = serving.poisson_requests(5, 50.0, 3, n_hi=300, step_scale=0.01)
  assert [r.arrival for r in a] == [r.arrival for r in b]
  assert [r.n_steps for r in a] == [r.n_steps for r in b]
  assert all(np.diff([r.arrival for r in a]) > 0)


def test_cohorts_are_never_rebuilt_and_state_stays_put():
  # each admission wave becomes one cohort batch; running cohorts are never
  # rebuilt or reloaded (set_full_state is never called), their state is read
  # only when one of their requests finishes, and every request still gets
  # exactly its steps
  clk = Clock()
  built = []

  class NoReload(FakeBatch):
    def set_full_state(self, *a, **k):
      raise AssertionError("a running cohort's state was reloaded")

    set_state = set_full_state

  def factory(systems, **kw):
    built.append(len(systems))
    return NoReload(systems, **kw)

  srv = serving.Server(chunk=10, clock=clk, batch_factory=factory)
  reqs = [_req(i, 10, steps, 0.0) for i, steps in enumerate((10, 20, 30, 40))]
  reqs += [_req(4, 10, 15, 0.05), _req(5, 10, 25, 0.05)]
  orig_tick = srv.tick

  def tick():
    clk.t += 0.01
    return orig_tick()

  srv.tick = tick
  res = srv.run(reqs, sleep=clk.sleep)
  for r in reqs:
    assert res[r.rid].error is None and res[r.rid].steps == r.n_steps
    np.testing.assert_allclose(res[r.rid].momentum, r.n_steps)
  assert built == [4, 2]
  rep = srv.report()
  assert rep["cohorts"] == 2 and rep["readbacks"] <= len(reqs)


def test_tick_lengths_come_from_a_small_set():
  seen = set()
  for limit in range(1, 200):
    n = serving._tick_steps(50, limit)
    assert 1 <= n <= min(50, limit)
    seen.add(n)
  assert seen <= {50, 25, 10, 5, 1}


def test_ended_systems_are_retired_in_their_cohort():
  # a finished request's system stops costing work at once: the cohort
  # retires it, and the cohort's other systems carry on unaffected
  clk = Clock()
  made = []

  def factory(systems, **kw):
    made.append(FakeBatch(systems, **kw))
    return made[-1]

  srv = serving.Server(chunk=10, clock=clk, batch_factory=factory)
  reqs = [_req(0, 10, 10, 0.0), _req(1, 10, 30, 0.0), _req(2, 10, 20, 0.0)]
  res = srv.run(reqs, sleep=clk.sleep)
  assert len(made) == 1
  assert made[0].retired == [0, 2]  # the last one ends with its cohort
  for r in reqs:
    assert res[r.rid].steps == r.n_steps
    np.testing.assert_allclose(res[r.rid].momentum, r.n_steps)
  np.testing.assert_allclose(made[0].p[:10], 10)   # not stepped after retirement
  np.testing.assert_allclose(made[0].p[20:], 20)
