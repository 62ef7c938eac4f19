"""The device-side wait of the fused Born finalize is bounded: a system whose
descreening items never all arrive (the test hook raises the count its
finalize chunks wait for) is flagged PB2_STATUS_WAIT_TIMEOUT after about a
second, the other systems' forces are exact, and once released the batch
computes every system exactly again.  Nothing here faults or hangs the GPU:
the wait gives up by itself."""

import time

import numpy as np
import pytest

from prolix_b200 import _lib, engine, synth

pytestmark = pytest.mark.gpu


def _fresh_forces(b, pos):
  b.set_positions(pos)  # invalidates the cached forces: a new evaluation
  return b.forces()


def test_finalize_wait_runs_out_flags_the_system_and_leaves_the_others_exact():
  systems = [synth.make_chain(n, 900 + n, compact=True) for n in (120, 70, 150)]
  with engine.Batch(systems) as b:
    b.set_fusion(_lib.FUSE_BONDED | _lib.FUSE_FINALIZE)
    pos = np.concatenate([s["positions"] for s in systems])
    ref = _fresh_forces(b, pos)
    assert not np.any(b.status(clear=True))
    b._check(b.lib.pb2_test_hold_system(b.handle, 1, 1))
    t0 = time.perf_counter()
    held = _fresh_forces(b, pos)
    waited = time.perf_counter() - t0
    st = b.status(clear=True)
    assert st[1] & _lib.STATUS_WAIT_TIMEOUT
    assert not (st[0] | st[2])
    lo, hi = b.offsets[1], b.offsets[2]
    np.testing.assert_array_equal(held[:lo], ref[:lo])
    np.testing.assert_array_equal(held[hi:], ref[hi:])
    assert waited < 30.0
    b._check(b.lib.pb2_test_hold_system(b.handle, 1, 0))
    np.testing.assert_array_equal(_fresh_forces(b, pos), ref)
    assert not np.any(b.status(clear=True))
