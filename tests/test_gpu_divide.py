"""The integrator's FP64 division by the mass (a reciprocal per atom and
two Markstein corrections) against CUDA's correctly rounded division, bit
for bit, on seeded operand pairs: random momenta of any sign and magnitude
against masses of 0.5-512 amu, plus masses with all-ones and all-zeros
significands, exact multiples, zeros and quotients in the subnormal range.
The end-to-end consequence (BAOAB steps bit-identical to the NumPy oracle)
is covered by the integrator parity tests."""

import ctypes

import pytest

from prolix_b200 import engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 20261203])
def test_markstein_division_equals_the_correctly_rounded_quotient(seed):
  ctx = engine.Context.get(0)
  bad = ctypes.c_longlong(-1)
  ex = (ctypes.c_double * 2)()
  ctx.check(ctx.lib.pb2_diag_div_check(ctx.handle, 1 << 30, seed, ctypes.byref(bad), ex))
  assert bad.value == 0, f"first mismatch at p={ex[0]!r}, m={ex[1]!r}"
