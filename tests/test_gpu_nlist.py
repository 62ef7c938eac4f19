"""Cell-list neighbour lists (jax_md layout) against brute force."""

import numpy as np
import pytest

from oracle import nlist as onl
from prolix_b200 import _lib, engine, synth

pytestmark = pytest.mark.gpu


def _check_rows(rows, systems, reach, tol=1e-3):
  off = 0
  for s in systems:
    n = len(s["charges"])
    tight = onl.neighbour_sets(s["positions"], reach - tol)
    loose = onl.neighbour_sets(s["positions"], reach + tol)
    for i in range(n):
      row = rows[off + i]
      got = row[row != n]
      assert len(got) == len(set(got.tolist())), "duplicate neighbour"
      g = set(got.tolist())
      assert tight[i] <= g <= loose[i], (i, len(tight[i]), len(g), len(loose[i]))
    off += n


def test_cell_list_matches_brute_force_ragged():
  systems = [synth.make_chain(n, 300 + k, compact=True) for k, n in enumerate([70, 640, 1500])]
  with engine.Batch(systems, cutoff=8.0, skin=2.0) as b:
    b.nl_build()
    rows = b.nl_get()
    assert b.nl_capacity() == rows.shape[1]
    rows2 = b.nl_get()
    b.nl_build()
    rows3 = b.nl_get()
  _check_rows(rows, systems, 10.0)
  np.testing.assert_array_equal(rows2, rows3)  # deterministic order
  # symmetric: j in row i <=> i in row j
  off = 0
  for s in systems:
    n = len(s["charges"])
    sets = [set(r[r != n].tolist()) for r in rows[off:off + n]]
    for i in range(n):
      for j in sets[i]:
        assert i in sets[j]
    off += n


def test_long_reach_rows_match_brute_force():
  # reach 16 A against 32-atom blocks of a compact chain: many blocks lie
  # wholly within reach of a warp's four rows and are stored without their
  # distances, beside blocks that are tested atom by atom
  systems = [synth.make_chain(n, 410 + k, compact=True) for k, n in enumerate([3000, 777])]
  with engine.Batch(systems, cutoff=14.0, skin=2.0) as b:
    b.nl_build()
    rows = b.nl_get()
    b.nl_build()
    again = b.nl_get()
  np.testing.assert_array_equal(rows, again)
  _check_rows(rows, systems, 16.0)
  off = 0
  for s in systems:
    n = len(s["charges"])
    for r in rows[off:off + n]:
      got = r[r != n]
      assert (r[len(got):] == n).all()  # sentinels after the neighbours
    off += n


def test_large_build_matches_brute_force():
  # 469 blocks: more two-row units than one wave of resident warps holds on
  # a B200, so the build takes four-row units (the smaller builds of the
  # other tests take two-row ones)
  s = synth.make_chain(15000, 77, compact=True)
  with engine.Batch([s], cutoff=9.0, skin=2.0) as b:
    b.nl_build()
    rows = b.nl_get()
  _check_rows(rows, [s], 11.0)


def test_capacity_not_a_multiple_of_four():
  # an odd fixed capacity: the sentinels go one slot at a time
  s = synth.make_chain(500, 12, compact=True)
  out = []
  for cap in (None, 501):
    kw = {} if cap is None else dict(nl_capacity=cap)
    with engine.Batch([s], cutoff=9.0, skin=2.0, **kw) as b:
      b.nl_build()
      out.append(b.nl_get())
  auto, odd = out
  assert odd.shape[1] == 501
  for ra, ro in zip(auto, odd):
    got = ro[ro != 500]
    np.testing.assert_array_equal(got, ra[ra != 500])
    assert (ro[len(got):] == 500).all()


def test_skin_rebuild_rule():
  s = synth.make_chain(500, 8, compact=True)
  with engine.Batch([s], cutoff=9.0, skin=2.0) as b:
    assert b.nl_check() == 1  # first call builds
    pos = s["positions"].copy()
    pos[7] += np.array([0.6, 0.0, 0.0])  # below skin/2
    b.set_positions(pos)
    assert b.nl_check() == 0
    pos[7] += np.array([0.6, 0.0, 0.0])  # now 1.2 A > skin/2
    b.set_positions(pos)
    assert b.nl_check() == 1
    rows = b.nl_get()
  _check_rows(rows, [dict(s, positions=pos)], 11.0)


def test_fixed_capacity_overflow_is_reported():
  s = synth.make_chain(800, 9, compact=True)
  with engine.Batch([s], cutoff=9.0, skin=2.0, nl_capacity=16) as b:
    with pytest.raises(_lib.PB2Error) as e:
      b.nl_build()
    assert e.value.code == -4
    assert b.status()[0] & _lib.STATUS_NLOVERFLOW


def test_neighbour_list_needs_a_cutoff():
  s = synth.make_chain(50, 1)
  with engine.Batch([s]) as b:
    with pytest.raises(_lib.PB2Error):
      b.nl_build()


@pytest.mark.parametrize("cutoffs", [dict(cutoff=9.0), dict(cutoff=8.0, gb_cutoff=12.0),
                                     dict(cutoff=10.0, born_cutoff=7.0)])
def test_pair_list_steps_equal_the_unlisted_steps(cutoffs):
  # the pair kernels on the skin-buffered block-pair list give the same bits
  # as scanning every block pair; a small skin makes the list rebuild often
  # during the run (a list that missed a rebuild would drop pairs)
  systems = synth.make_batch(5, 77, 300, 1500, compact=True, **synth.PHYSICAL_RANGES)
  fields = ("position", "momentum", "force")
  out = []
  for pl in (True, False):
    with engine.Batch(systems, skin=0.2, pair_list=pl, dt=engine.akma_dt(2.0),
                      kT=600 * engine.KB_KCAL, **cutoffs) as b:
      e0, f0 = b.energy_forces()
      b.langevin_init()
      b.langevin_run(120)
      st = b.get_state(fields=fields)
      out.append((e0, f0, st))
  (ea, fa, sa), (eb, fb, sb) = out
  np.testing.assert_array_equal(fa, fb)
  np.testing.assert_array_equal(ea, eb)
  for f in fields:
    np.testing.assert_array_equal(sa[f], sb[f])
  assert np.isfinite(sa["position"]).all()


def test_asynchronous_check_rebuilds_on_the_device():
  # the check and the rebuild it triggers are enqueued without a host wait;
  # a list that outgrows its rows is grown at the next host visit (nl_get)
  s = synth.make_chain(900, 14, compact=True)
  with engine.Batch([s], cutoff=6.0, skin=1.0) as b:
    b.nl_build()
    cap0 = b.nl_capacity()
    assert b.nl_last_build_ms() > 0.0
    pos = s["positions"] * 0.8  # compress: every atom moves well past skin/2, rows grow
    b.set_positions(pos)
    assert b.nl_check(wait=False) is None
    rows = b.nl_get()
    assert b.nl_capacity() >= cap0
  _check_rows(rows, [dict(s, positions=pos)], 7.0)
