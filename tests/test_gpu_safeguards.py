"""Safeguards of prolix's batched Langevin step (batched_simulate.py:218-382)
on the CUDA path, against the oracle's restatement: speed limit,
displacement cap, closing-force cap and the per-system warn counts
(typing.py:559-563)."""

import numpy as np
import pytest
import torch

from oracle import bonded
from oracle import integrator as ointeg
from oracle import prng
from prolix_b200 import engine, streamed, synth
from prolix_b200._lib import USE_BONDED, USE_CMAP

pytestmark = pytest.mark.gpu

DT, KT, GAMMA = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)


def test_settings_and_zero_counts():
  systems = [synth.make_chain(n, n, compact=True) for n in (60, 90, 75)]
  with engine.Batch(systems) as b:
    assert b.safeguards() == {"vlimit": 0.0, "max_dx": 0.0, "force_cap": 0.0}
    b.set_safeguards(**engine.BATCHED_SAFEGUARDS)
    assert b.safeguards() == engine.BATCHED_SAFEGUARDS
    b.set_safeguards(vlimit=-1.0, max_dx=0.5)  # <= 0 turns a limit off
    assert b.safeguards() == {"vlimit": 0.0, "max_dx": 0.5, "force_cap": 0.0}
    with pytest.raises(RuntimeError):
      b.set_safeguards(vlimit=float("nan"))
    c = b.warn_counts()
    assert c.shape == (3, 4) and c.dtype == np.int32 and not c.any()


def test_zero_force_steps_match_the_oracle_bit_for_bit():
  # F = 0: speed and displacement limits firing on some steps; positions,
  # momenta, keys and counts equal the FP64 restatement exactly, per system
  keys = [prng.prng_key(1234), prng.prng_key(77)]
  systems = [dict(synth.make_chain(97, 21, compact=True), key=keys[0]),
             dict(synth.make_chain(64, 5, compact=True), key=keys[1])]
  guards = (1.6, 0.03, 0.0)
  with engine.Batch(systems, terms=0, dt=DT, kT=KT, gamma=GAMMA) as b:
    b.set_safeguards(*guards)
    b.langevin_init()
    b.langevin_run(5)
    b.langevin_run(4)
    st = b.get_state()
    counts = b.warn_counts()
  zero = lambda r: np.zeros_like(r)
  for k, s in enumerate(systems):
    lo, hi = b.offsets[k], b.offsets[k + 1]
    o = ointeg.init(zero, keys[k], s["positions"], s["masses"], KT)
    oc = np.zeros(4, np.int64)
    o = ointeg.run(o, zero, 9, DT, KT, GAMMA, guards=guards, counts=oc)
    np.testing.assert_array_equal(st["position"][lo:hi], o.position)
    np.testing.assert_array_equal(st["momentum"][lo:hi], o.momentum)
    np.testing.assert_array_equal(st["key"][k], o.key)
    assert counts[k].tolist() == oc.tolist()
  assert counts[:, 0].sum() > 0 and counts[:, 3].sum() > 0  # both limits fired


def test_force_cap_tracks_the_oracle():
  # bonded forces above a low cap: the closing force is capped, the initial
  # force opens the first step as it is
  s = synth.make_chain(120, 8, compact=True, cmap=True)
  guards = (0.0, 0.0, 25.0)
  key = prng.prng_key(99)
  with engine.Batch([s], terms=USE_BONDED | USE_CMAP, key=key, dt=DT, kT=KT, gamma=GAMMA) as b:
    b.set_safeguards(*guards)
    b.langevin_init()
    b.langevin_run(20)
    st = b.get_state()
    counts = b.warn_counts(reset=True)
    assert not b.warn_counts().any()
  force = lambda r: bonded.bonded_all(s, r)[1]
  o = ointeg.init(force, key, s["positions"], s["masses"], KT)
  oc = np.zeros(4, np.int64)
  o = ointeg.run(o, force, 20, DT, KT, GAMMA, guards=guards, counts=oc)
  np.testing.assert_allclose(st["position"], o.position, rtol=0, atol=1e-8)
  np.testing.assert_allclose(st["momentum"], o.momentum, rtol=0, atol=1e-7)
  assert 0 < oc[1] and counts[0].tolist() == oc.tolist()


def test_graph_chunks_and_host_round_trips_equal_one_run():
  # chunk boundaries (the closing force capped by the finish launch, then
  # opening the next chunk) and host round trips change nothing
  systems = synth.make_batch(3, 12, 80, 160, compact=True, **synth.PHYSICAL_RANGES)
  guards = (1.2, 0.025, 40.0)
  fields = ("position", "momentum", "force")
  with engine.Batch(systems, graph_chunk=4) as g, engine.Batch(systems) as e, \
       engine.Batch(systems) as h:
    for b in (g, e, h):
      b.set_safeguards(*guards)
      b.langevin_init()
    e.set_profiling(True)  # eager launches, no graphs
    g.langevin_run(10)
    e.langevin_run(10)
    st = h.get_state(fields=fields)
    host = {f: streamed.pinned(st[f].shape) for f in fields}
    for f in fields:
      host[f][...] = st[f]
    for n in (3, 3, 4):
      h.langevin_run_host(host["position"], host["momentum"], host["force"], n)
    torch.cuda.synchronize()
    sg, se = g.get_state(), e.get_state()
    for f in fields:
      assert np.array_equal(sg[f], se[f]), f
      assert np.array_equal(host[f], sg[f]), f
    cg = g.warn_counts()
    assert np.array_equal(cg, e.warn_counts()) and np.array_equal(cg, h.warn_counts())
    assert cg[:, 0].sum() > 0 and cg[:, 1].sum() > 0 and cg[:, 3].sum() > 0
