"""The committed golden fixtures (tests/golden, written by make_golden.py):
the seeded generator still produces the same inputs and the FP64 oracle
still produces the same outputs."""

import importlib.util
import os

import numpy as np
import pytest

from oracle import energy

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_maker():
  spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
  mod = importlib.util.module_from_spec(spec)
  spec.loader.exec_module(mod)
  return mod


MG = load_maker()
FIX = np.load(os.path.join(GOLDEN, "oracle_small.npz"))


@pytest.mark.parametrize("name", [c[0] for c in MG.CASES])
def test_oracle_reproduces_the_fixture(name):
  s, cutoff = MG.case_system(name)
  assert str(FIX[f"{name}/positions_digest"]) == MG.positions_digest(s["positions"])
  e, f, ex = energy.energy_forces(s, s["positions"], cutoff)
  terms = np.array([e[t] for t in energy.TERMS + ("total",)])
  assert list(FIX["term_names"]) == list(energy.TERMS + ("total",))
  np.testing.assert_allclose(terms, FIX[f"{name}/terms"], rtol=1e-10, atol=1e-10)
  np.testing.assert_allclose(f, FIX[f"{name}/forces"], rtol=1e-10, atol=1e-10)
  np.testing.assert_allclose(ex["born_radii"], FIX[f"{name}/born_radii"], rtol=1e-12)


def test_zero_force_trajectory_reproduces_the_fixture():
  s, st = MG.zero_force_run()
  name = MG.ZERO_FORCE[0]
  assert str(FIX[f"{name}/positions_digest"]) == MG.positions_digest(s["positions"])
  np.testing.assert_array_equal(st.position, FIX[f"{name}/position"])
  np.testing.assert_array_equal(st.momentum, FIX[f"{name}/momentum"])
  np.testing.assert_array_equal(st.key, FIX[f"{name}/key"])
