"""Stand-in for ``jax.scipy`` (TEST INFRASTRUCTURE ONLY)."""

from . import special  # noqa: F401
