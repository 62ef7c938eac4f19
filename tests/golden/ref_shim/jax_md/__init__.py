"""Stand-in for the few jax-md 0.2.27 pieces prolix's force-field files call.

TEST INFRASTRUCTURE ONLY.  jax-md is a third-party dependency of prolix
(uv.lock pins 0.2.27) and is not installed here; the functions below restate
its published definitions (jax_md/space.py ``free``, ``distance``;
jax_md/energy.py ``simple_spring``, ``simple_spring_bond``; jax_md/smap.py
``bond``) in NumPy.
"""

from . import energy, partition, space, util  # noqa: F401
