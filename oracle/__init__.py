"""FP64 CPU restatement of prolix's implicit-solvent MD step (the oracle).

TEST INFRASTRUCTURE ONLY.  Nothing in the ``prolix_b200`` package imports or
calls this package: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it, and only as the checker or the CPU
baseline, never as the thing measured on the GPU.

Parity status: the physics formulas follow the reference files cited in each
function; they are pinned by the reference's own analytic known-answer tests
(Born ion, dense == complete neighbour list, finite-difference gradients,
NVE drift) restated in ``tests/test_oracle_*.py``.  The threefry2x32 block is
pinned by the Random123 known-answer vectors; the exact ``jax.random`` bit
streams built on top of it (key split layout, normal sampling) are restated
from JAX's published algorithm and are "parity unpinned" (no JAX here).
The reference's own JAX code cannot run here (JAX absent), so no output of
the reference itself pins the oracle.
"""
