"""Explicit 1-4 exception pairs on the CUDA path (prolix bonded.py:186-230,
system.py:149-159) against the oracle."""

import types

import numpy as np
import pytest

from oracle import energy as oenergy
from prolix_b200 import engine, synth
from prolix_b200 import system as psys
from prolix_b200._lib import TERM_NAMES, USE_ALL, USE_BONDED, USE_LJ
from test_exceptions_cpu import with_explicit_14

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
  return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_exception_pairs_match_the_oracle():
  s = with_explicit_14(synth.make_chain(166, 2, compact=True, cmap=True), sigma_jitter=0.1)
  e_ref, f_ref, _ = oenergy.energy_forces(s, s["positions"])
  with engine.Batch([s]) as b:
    e, f = b.energy_forces()
  for k, name in enumerate(TERM_NAMES):
    assert abs(e[0, k] - e_ref[name]) <= 1e-6 * abs(e_ref[name]) + 1e-6, name
  assert e_ref["exception"] != 0.0
  assert rel_rms(f, f_ref) < 1e-5


def test_explicit_and_scaled_14_agree_on_the_gpu():
  s = synth.make_chain(300, 6, compact=True)
  ex = with_explicit_14(s)
  with engine.Batch([s, ex]) as b:
    e, f = b.energy_forces()
  lo = b.offsets[1]
  i_lj, i_c, i_x, i_t = (TERM_NAMES.index(t) for t in ("lj", "coulomb", "exception", "total"))
  assert e[0, i_x] == 0.0 and e[1, i_x] != 0.0
  a, c = e[0, i_lj] + e[0, i_c], e[1, i_lj] + e[1, i_c] + e[1, i_x]
  assert abs(a - c) <= 1e-6 * abs(a)
  assert abs(e[0, i_t] - e[1, i_t]) <= 1e-6 * abs(e[0, i_t])
  assert rel_rms(f[lo:], f[:lo]) < 1e-6


def test_exception_terms_follow_the_term_bits():
  s = with_explicit_14(synth.make_chain(120, 9, compact=True))
  from oracle import bonded
  ref_lj, _ = bonded.exception_pairs(s["positions"], s["exception_pairs"], s["exception_sigmas"],
                                     s["exception_epsilons"], np.zeros(len(s["exception_pairs"])))
  with engine.Batch([s], terms=USE_LJ) as b:
    e, _ = b.energy_forces()
  assert abs(e[0, TERM_NAMES.index("exception")] - ref_lj) <= 1e-6 * abs(ref_lj) + 1e-6
  with engine.Batch([s], terms=USE_BONDED) as b:
    e, _ = b.energy_forces()
  assert e[0, TERM_NAMES.index("exception")] == 0.0


def test_make_energy_fn_takes_exceptions_from_the_exclusion_spec():
  s = synth.make_chain(140, 4, compact=True)
  ex = with_explicit_14(s)
  spec = types.SimpleNamespace(
      idx_12_13=ex["excl_pairs"], idx_14=np.zeros((0, 2), np.int32),
      scale_14_elec=0.83333333, scale_14_vdw=0.5,
      exception_pairs=ex["exception_pairs"], exception_sigmas=ex["exception_sigmas"],
      exception_epsilons=ex["exception_epsilons"], exception_chargeprods=ex["exception_chargeprods"])
  sysd = {k: v for k, v in s.items() if k not in ("excl_pairs", "excl_kind")}
  terms = psys.make_energy_fn(None, sysd, cutoff_distance=0.0, implicit_solvent=True,
                              return_decomposed=True, exclusion_spec=spec)
  e_ref, _, _ = oenergy.energy_forces(ex, ex["positions"])
  got = terms["exception"](s["positions"])
  assert abs(got - e_ref["exception"]) <= 1e-6 * abs(e_ref["exception"])
  assert abs(terms["total"](s["positions"]) - e_ref["total"]) <= 1e-6 * abs(e_ref["total"])
