"""Loader for the host C helper library (``libpb2_host.so``)."""

from __future__ import annotations

import ctypes
import threading

from . import _build

_LOCK = threading.Lock()
_LIB = None


def lib() -> ctypes.CDLL:
  global _LIB
  with _LOCK:
    if _LIB is None:
      path = _build.HOST_LIB
      if not path.exists():
        _build.build_host()
      h = ctypes.CDLL(str(path))
      dp = ctypes.POINTER(ctypes.c_double)
      h.pb2_synth_grow_chain.restype = ctypes.c_int
      h.pb2_synth_grow_chain.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double,
                                         ctypes.c_ulonglong, dp, dp]
      _LIB = h
  return _LIB
