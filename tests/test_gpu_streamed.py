"""Host-resident state: pb2_langevin_run_host, and the same systems split
into groups on their own streams (prolix_b200.streamed)."""

import numpy as np
import pytest
import torch

from prolix_b200 import engine, streamed, synth

pytestmark = pytest.mark.gpu


def _systems():
  return synth.make_batch(7, 31, 40, 300, compact=True, **synth.PHYSICAL_RANGES)


def test_run_host_matches_device_state_path():
  # state in from host arrays, steps, state out: the same bits as
  # pb2_set_full_state + pb2_langevin_run + pb2_get_state, over two calls
  systems = _systems()
  fields = ("position", "momentum", "force")
  with engine.Batch(systems) as a, engine.Batch(systems) as b:
    a.langevin_init()
    b.langevin_init()
    st = a.get_state(fields=fields)
    host = {f: streamed.pinned(st[f].shape) for f in fields}
    for f in fields:
      host[f][...] = st[f]
    for _ in range(2):
      b.langevin_run_host(host["position"], host["momentum"], host["force"], 3)
      torch.cuda.synchronize()
      a.set_full_state(st["position"], st["momentum"], st["force"])
      a.langevin_run(3)
      st = a.get_state(fields=fields)
      for f in fields:
        assert np.array_equal(host[f], st[f]), f


def test_grouped_streams_match_one_batch():
  systems = _systems()
  fields = ("position", "momentum", "force")
  with engine.Batch(systems) as one, streamed.StreamedEnsemble(systems, groups=3) as ens:
    assert len(ens.batches) == 3
    one.langevin_init()
    ens.langevin_init()
    ref = one.get_state(fields=fields)
    st = ens.get_state()
    for f in fields:
      assert np.array_equal(st[f], ref[f]), f
    for _ in range(2):
      ens.run_host(st["position"], st["momentum"], st["force"], 4)
      one.langevin_run(4)
    ref = one.get_state(fields=fields)
    for f in fields:
      assert np.array_equal(st[f], ref[f]), f
    assert np.all(np.isfinite(st["position"]))


def test_run_host_rejects_arrays_it_cannot_write_in_place():
  systems = _systems()[:2]
  with engine.Batch(systems) as b:
    b.langevin_init()
    n = b.n_atoms
    good = np.zeros((n, 3))
    with pytest.raises(ValueError):
      b.langevin_run_host(good, good, np.zeros((n, 3), dtype=np.float32), 1)
    with pytest.raises(ValueError):
      b.langevin_run_host(good, good, np.zeros((3, n)).T, 1)
