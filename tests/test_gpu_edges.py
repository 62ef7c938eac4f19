"""Edge cases of the batch: block-boundary and tiny system sizes in one
ragged batch (two i-blocks per warp, lone last blocks, partial j-blocks),
term subsets (the kernels' generic variant) summing to the full force, and
input validation through the C ABI."""

import numpy as np
import pytest

from oracle import energy as oenergy
from prolix_b200 import _lib, engine, synth
from prolix_b200._lib import USE_BONDED, USE_CMAP, USE_COULOMB, USE_GB, USE_LJ

pytestmark = pytest.mark.gpu


def test_block_boundary_sizes_in_one_batch():
  sizes = (1, 2, 3, 31, 32, 33, 63, 64, 65, 97, 128, 129)
  systems = [synth.make_chain(n, 700 + n, compact=True) for n in sizes]
  with engine.Batch(systems) as b:
    e, f = b.energy_forces()
    parts = b.split(f)
  for k, (s, fk) in enumerate(zip(systems, parts)):
    e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"])
    scale = max(np.linalg.norm(f_ref), 1e-3)
    assert np.linalg.norm(fk - f_ref) / scale < 1e-5, sizes[k]
    assert abs(e[k][-1] - e_ref["total"]) <= 1e-6 * abs(e_ref["total"]) + 1e-5, sizes[k]


def test_term_subsets_add_up_to_the_full_force():
  systems = [synth.make_chain(n, 800 + n, compact=True, cmap=True) for n in (166, 257)]
  with engine.Batch(systems) as b:
    e_all, f_all = b.energy_forces()
  total_f = np.zeros_like(f_all)
  for terms in (USE_BONDED, USE_CMAP, USE_LJ, USE_COULOMB, USE_GB, USE_LJ | USE_GB):
    with engine.Batch(systems, terms=terms) as b:
      e, f = b.energy_forces()
    if terms != USE_LJ | USE_GB:
      total_f += f
    for t, name in enumerate(_lib.TERM_NAMES[:-1]):
      if e[0][t] != 0.0:  # a term that is on matches the all-terms evaluation
        np.testing.assert_allclose(e[:, t], e_all[:, t], rtol=1e-12, atol=1e-9)
  rel = np.linalg.norm(total_f - f_all) / np.linalg.norm(f_all)
  assert rel < 1e-6


def _bad(system, match, **kw):
  with pytest.raises((_lib.PB2Error, ValueError), match=match):
    engine.Batch([system], **kw).close()


def test_invalid_inputs_are_rejected():
  s = synth.make_chain(100, 3)
  _bad(dict(s, masses=np.where(np.arange(100) == 7, 0.0, s["masses"])), "masses")
  _bad(dict(s, bonds=np.array([[0, 1], [5, 100]])), "index")
  _bad(dict(s, excl_pairs=np.array([[4, 2]]), excl_kind=np.array([0])), "i < j")
  # atom 0 with exclusion partners in seventeen different 32-atom blocks of
  # the input order (a spatial order may gather them into fewer blocks, and
  # is then accepted)
  n = 600
  far = dict(synth.make_chain(n, 4), excl_pairs=np.array([[0, 33 * k + 1] for k in range(17)]),
             excl_kind=np.zeros(17, np.int32))
  _bad(far, "more than 16", keep_atom_order=True)
  with pytest.raises(ValueError):
    engine.Batch([])
