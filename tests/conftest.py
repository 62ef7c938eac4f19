import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)


def pytest_configure(config):
  config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the CUDA library")
  config.addinivalue_line("markers", "slow: long-running")


def gpu_available() -> bool:
  try:
    import torch
    return torch.cuda.is_available()
  except Exception:
    return False
