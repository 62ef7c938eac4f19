"""The allocation-free Born-radius entry point, checked against the regular
batch entry point and against the FP64 oracle.

pb2_born_radii_noalloc serves callers that cannot call cudaMalloc (an XLA
custom-call handler that may only use the buffers it is handed, code running
under CUDA stream capture, hosts with a fixed memory pool).  Its scratch is a
static device array shared by all calls, so the check runs it twice in a row
on different systems: a second call must not see the first call's sums.
This file is collected last so a failure here comes after every other test.
"""

import ctypes

import numpy as np
import pytest

from oracle import gbsa as ogbsa
from prolix_b200 import engine, synth

pytestmark = pytest.mark.gpu

MAX_ATOMS = 32768


def _noalloc_born(ctx, system, cutoff=0.0):
  import torch
  dev = torch.device("cuda", 0)
  pos = torch.tensor(np.asarray(system["positions"]), dtype=torch.float64, device=dev).contiguous()
  rad = torch.tensor(np.asarray(system["radii"]), dtype=torch.float64, device=dev)
  sr = torch.tensor(np.asarray(system["scaled_radii"]), dtype=torch.float64, device=dev)
  out = torch.full((rad.numel(),), float("nan"), dtype=torch.float64, device=dev)
  torch.cuda.synchronize()
  rc = ctx.lib.pb2_born_radii_noalloc(ctx.handle, rad.numel(), pos.data_ptr(), rad.data_ptr(),
                                      sr.data_ptr(), float(cutoff), out.data_ptr(), None)
  ctx.check(rc)
  torch.cuda.synchronize()
  return out.cpu().numpy()


@pytest.mark.parametrize("cutoff", [0.0, 9.0])
def test_noalloc_born_radii_match_batch_entry_point(cutoff):
  ctx = engine.Context.get(0)
  systems = [synth.make_chain(700, 41, compact=True), synth.make_chain(166, 1)]
  for _ in range(2):  # two calls in a row per system, shared scratch
    for s in systems:
      got = _noalloc_born(ctx, s, cutoff)
      with engine.Batch([s], cutoff=cutoff) as b:
        ref = b.born_radii()
      np.testing.assert_allclose(got, ref, rtol=2e-6)
      oracle = ogbsa.born_radii(np.asarray(s["positions"]), np.asarray(s["radii"]),
                                np.asarray(s["scaled_radii"]), cutoff)[0]
      np.testing.assert_allclose(got, oracle, rtol=2e-6)


def test_noalloc_rejects_too_many_atoms():
  ctx = engine.Context.get(0)
  rc = ctx.lib.pb2_born_radii_noalloc(ctx.handle, MAX_ATOMS + 1, ctypes.c_void_p(8),
                                      ctypes.c_void_p(8), ctypes.c_void_p(8), 0.0,
                                      ctypes.c_void_p(8), None)
  assert rc == -1
  assert b"PB2_NOALLOC_MAX_ATOMS" in ctx.lib.pb2_last_error(ctx.handle)
