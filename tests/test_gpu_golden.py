"""The CUDA path against the committed golden fixtures (tests/golden):
per-term energies relative 1e-6 (+1e-6 kcal/mol), forces relative RMS
1e-5, Born radii 2e-6, and the zero-force BAOAB trajectory bit for bit."""

import numpy as np
import pytest

from oracle import prng
from prolix_b200 import engine
from prolix_b200._lib import TERM_NAMES
from test_golden_cpu import FIX, MG

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [c[0] for c in MG.CASES])
def test_gpu_matches_the_fixture(name):
  s, cutoff = MG.case_system(name)
  with engine.Batch([s], cutoff=cutoff) as b:
    e, f = b.energy_forces()
    born = b.born_radii()
  names = list(FIX["term_names"])
  ref = FIX[f"{name}/terms"]
  for k, t in enumerate(TERM_NAMES):
    r = ref[names.index(t)]
    assert abs(e[0, k] - r) <= 1e-6 * abs(r) + 1e-6, t
  fr = FIX[f"{name}/forces"]
  assert np.linalg.norm(f - fr) / np.linalg.norm(fr) < 1e-5
  np.testing.assert_allclose(born, FIX[f"{name}/born_radii"], rtol=2e-6)


def test_zero_force_trajectory_is_the_fixture():
  name, n, seed, kseed, steps = MG.ZERO_FORCE
  s = MG.synth.make_chain(n, seed, compact=True)
  with engine.Batch([s], terms=0, key=prng.prng_key(kseed), dt=engine.akma_dt(1.0),
                    kT=300 * engine.KB_KCAL, gamma=engine.akma_gamma(1.0)) as b:
    b.langevin_init()
    b.langevin_run(steps)
    st = b.get_state()
  np.testing.assert_array_equal(st["position"], FIX[f"{name}/position"])
  np.testing.assert_array_equal(st["momentum"], FIX[f"{name}/momentum"])
  np.testing.assert_array_equal(st["key"][0], FIX[f"{name}/key"])
