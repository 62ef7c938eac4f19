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


def test_run_device_matches_device_state_path():
  # the jax.ffi form: caller-owned device arrays in and out, on one stream
  systems = _systems()
  fields = ("position", "momentum", "force")
  with engine.Batch(systems) as a, engine.Batch(systems) as b:
    a.langevin_init()
    b.langevin_init()
    st = a.get_state(fields=fields)
    dev = {f: torch.tensor(st[f], device="cuda") for f in fields}
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
      b.langevin_run_device(dev["position"].data_ptr(), dev["momentum"].data_ptr(),
                            dev["force"].data_ptr(), 3, stream)
      torch.cuda.synchronize()
      a.set_full_state(st["position"], st["momentum"], st["force"])
      a.langevin_run(3)
      st = a.get_state(fields=fields)
      for f in fields:
        assert np.array_equal(dev[f].cpu().numpy(), st[f]), f


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


def test_spatial_atom_order_is_invisible_to_the_caller():
  # the batch stores each system's atoms in a spatial order by default; every
  # array that crosses the interface stays in the caller's order, so the two
  # layouts give the same forces (to float32 summation order), energies,
  # Born radii and, after steps, the same trajectory to within rounding
  systems = synth.make_batch(3, 77, 300, 900, compact=True, **synth.PHYSICAL_RANGES)
  with engine.Batch(systems) as a, engine.Batch(systems, keep_atom_order=True) as b:
    ea, fa = a.energy_forces()
    eb, fb = b.energy_forces()
    np.testing.assert_allclose(ea, eb, rtol=1e-9, atol=1e-6)
    assert np.linalg.norm(fa - fb) / np.linalg.norm(fb) < 1e-6
    np.testing.assert_allclose(a.born_radii(), b.born_radii(), rtol=1e-6)
    a.langevin_init()
    b.langevin_init()
    a.langevin_run(20)
    b.langevin_run(20)
    xa = a.get_state(fields=("position",))["position"]
    xb = b.get_state(fields=("position",))["position"]
    assert np.max(np.abs(xa - xb)) < 1e-4


def test_queued_round_trips_without_host_waits():
  # several host round trips queued back to back (each step copies the state
  # in from and out to the same host arrays) give the state of the same
  # steps run on the device alone
  systems = _systems()
  fields = ("position", "momentum", "force")
  with engine.Batch(systems) as one, streamed.StreamedEnsemble(systems, groups=3) as ens:
    one.langevin_init()
    ens.langevin_init()
    st = ens.get_state()
    ens.synchronize()
    for _ in range(4):
      ens.run_host(st["position"], st["momentum"], st["force"], 2, wait=False)
    ens.synchronize()
    one.langevin_run(8)
    ref = one.get_state(fields=fields)
    for f in fields:
      assert np.array_equal(st[f], ref[f]), f


def test_round_trip_of_zero_steps_leaves_the_state():
  # copies in and out with no step between: x, p and F come back bit for bit
  # (fixed point -> FP64 -> fixed point is exact for the forces)
  systems = _systems()[:3]
  with engine.Batch(systems) as b:
    b.langevin_init()
    b.langevin_run(2)
    st = b.get_state(fields=("position", "momentum", "force"))
    host = {f: streamed.pinned(st[f].shape) for f in st}
    for f in st:
      host[f][...] = st[f]
    b.langevin_run_host(host["position"], host["momentum"], host["force"], 0)
    torch.cuda.synchronize()
    for f in st:
      assert np.array_equal(host[f], st[f]), f
