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
