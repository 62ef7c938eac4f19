"""Loads prolix's own force-field source files, unmodified, on the NumPy
stand-in for JAX in ``ref_shim/``.

TEST INFRASTRUCTURE ONLY: used by ``make_ref_fixtures.py`` to run the
reference in this container; nothing on the GPU box imports it.

The reference package is not installed (it needs JAX, jax-md, equinox and
proxide, none of which exist here).  Instead ``prolix``, ``prolix.physics``
and ``prolix.utils`` are registered as bare packages whose search path is
the reference source tree, so ``prolix.physics.generalized_born`` and the
other files load straight from it without running the package
``__init__`` files (which import the whole framework).  ``prolix.typing``
is the small stand-in in ``ref_shim/prolix_typing_stub.py``.
"""

from __future__ import annotations

import importlib
import importlib.util
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
DEFAULT_SRC = "/root/reference/src"

MODULES = ("generalized_born", "optimization", "bonded", "cmap", "neighbor_list", "tiling")


def load(src: str | None = None) -> dict:
  """Return {name: module} for the reference physics modules in MODULES."""
  src = src or os.environ.get("PROLIX_REFERENCE_SRC", DEFAULT_SRC)
  pkg_dir = os.path.join(src, "prolix")
  if not os.path.isdir(os.path.join(pkg_dir, "physics")):
    raise FileNotFoundError(f"prolix sources not found under {src}")
  if SHIM not in sys.path:
    sys.path.insert(0, SHIM)
  import jax  # noqa: F401  (the stand-in)
  if not hasattr(jax, "custom_vjp") or "ref_shim" not in jax.__file__:
    raise RuntimeError("a real jax is importable; the fixtures are made with the NumPy stand-in")

  for name, path in (("prolix", pkg_dir), ("prolix.physics", os.path.join(pkg_dir, "physics")),
                     ("prolix.utils", os.path.join(pkg_dir, "utils"))):
    if name not in sys.modules:
      m = types.ModuleType(name)
      m.__path__ = [path]
      sys.modules[name] = m
  if "prolix.typing" not in sys.modules:
    spec = importlib.util.spec_from_file_location("prolix.typing",
                                                  os.path.join(SHIM, "prolix_typing_stub.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    sys.modules["prolix.typing"] = m
    sys.modules["prolix"].typing = m
  return {name: importlib.import_module(f"prolix.physics.{name}") for name in MODULES}
