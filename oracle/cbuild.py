"""Builds the C restatement of the oracle (TEST INFRASTRUCTURE ONLY).

gcc -O3 -march=native -fopenmp on oracle/c/oracle_forces.c, output
oracle/liboracle_forces.so (git-ignored, travels with the tree).
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "c" / "oracle_forces.c"
LIB = HERE / "liboracle_forces.so"


def build(force: bool = False) -> Path:
  if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
    cc = shutil.which("gcc") or "cc"
    tmp = LIB.with_suffix(".so.tmp")
    # -march=x86-64-v3 rather than native: the library travels to other hosts
    subprocess.run([cc, "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", "-o", str(tmp),
                    str(SRC), "-lm"], check=True)
    os.replace(tmp, LIB)
  return LIB
