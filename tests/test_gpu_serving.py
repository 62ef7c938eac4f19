"""Continuous-batching server on the GPU: every result equals the same
request run alone (bit for bit), failures and cancellations stay local."""

import numpy as np
import pytest

from prolix_b200 import serving, synth

pytestmark = pytest.mark.gpu


def _requests():
  sizes = [180, 700, 90, 1200, 333]
  steps = [130, 60, 170, 90, 75]
  reqs = []
  for i, (n, k) in enumerate(zip(sizes, steps)):
    reqs.append(serving.Request(system=synth.make_chain(n, 500 + i, compact=True), n_steps=k,
                                key=(0, 1000 + i), arrival=0.03 * i, rid=i))
  return reqs


def _alone(req):
  srv = serving.Server(chunk=40)
  r = serving.Request(system=req.system, n_steps=req.n_steps, key=req.key, rid=req.rid)
  return srv.run([r])[req.rid]


def test_each_result_is_the_same_alone_and_in_the_mix():
  reqs = _requests()
  mixed = serving.Server(chunk=40).run(reqs)
  assert all(r.error is None for r in mixed.values())
  for req in reqs:
    a = _alone(req)
    m = mixed[req.rid]
    assert m.steps == req.n_steps == a.steps
    np.testing.assert_array_equal(m.position, a.position)
    np.testing.assert_array_equal(m.momentum, a.momentum)
    np.testing.assert_array_equal(m.key, a.key)


def test_non_finite_request_is_evicted_others_unchanged():
  reqs = _requests()[:3]
  bad = synth.make_chain(150, 77, compact=True)
  bad["positions"] = bad["positions"].copy()
  bad["positions"][5, 1] = np.nan
  reqs.append(serving.Request(system=bad, n_steps=50, key=(0, 9), arrival=0.01, rid=99))
  res = serving.Server(chunk=40).run(reqs)
  assert res[99].error is not None
  for req in reqs[:3]:
    np.testing.assert_array_equal(res[req.rid].position, _alone(req).position)


def test_budget_admission_and_cancellation():
  reqs = _requests()
  srv = serving.Server(chunk=40, max_batch_atoms=1300)  # at most ~1 large system at a time
  srv.cancel(2)
  res = srv.run(reqs)
  assert res[2].error == "cancelled"
  done = [r for r in res.values() if r.error is None]
  assert len(done) == 4
  rep = srv.report()
  assert rep["completed"] == 4 and rep["p99_s"] >= rep["p50_s"] > 0
  for req in reqs:
    if req.rid != 2:
      np.testing.assert_array_equal(res[req.rid].position, _alone(req).position)


@pytest.mark.parametrize("cutoff", [0.0, 12.0])
def test_retired_system_stops_and_the_rest_run_as_without_it(cutoff):
  # retire system 1 after 20 steps: it keeps its 20-step state through 30
  # more steps of the batch, and systems 0 and 2 end bit-identical to a
  # batch that never held it (the pair work list is compacted on the
  # device; at the cutoff, the pair list is rebuilt without it)
  from prolix_b200 import engine
  systems = [dict(synth.make_chain(n, 40 + n, compact=True), key=(0, 7 + n)) for n in (150, 400, 90)]

  def run(idx, plan):
    with engine.Batch([systems[i] for i in idx], cutoff=cutoff) as b:
      b.langevin_init()
      for n, retire in plan:
        b.langevin_run(n)
        for s in retire:
          b.retire(s)
      st = b.get_state(fields=("position", "momentum", "key"))
      return {f: [st[f][b.offsets[k]:b.offsets[k + 1]] if f != "key" else st[f][k]
                  for k in range(len(idx))] for f in st}

  mixed = run([0, 1, 2], [(20, [1]), (30, [])])
  alone02 = run([0, 2], [(50, [])])
  alone1 = run([1], [(20, [])])
  for f in ("position", "momentum", "key"):
    np.testing.assert_array_equal(mixed[f][0], alone02[f][0])
    np.testing.assert_array_equal(mixed[f][2], alone02[f][1])
    np.testing.assert_array_equal(mixed[f][1], alone1[f][0])
