"""In-tree build of the package's native libraries.

* ``libprolix_b200.so``: the CUDA kernels and the C ABI (nvcc, sm_100a only).
* ``libpb2_host.so``: host C helpers (synthetic chain growth).
* ``libprolix_b200_ffi.so`` (only on request): the XLA FFI handlers of
  ``csrc/ffi/pb2_ffi.cc``, which need the headers of an XLA / jaxlib
  install (``xla/ffi/api/ffi.h``): ``python -m prolix_b200._build --ffi
  <include dir>`` or ``PB2_XLA_FFI_INCLUDE=<include dir>``.  The default
  build skips it.

All land next to this file so they travel with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
CUDA_LIB = PKG / "libprolix_b200.so"
HOST_LIB = PKG / "libpb2_host.so"

CUDA_SOURCES = ["pb2_api.cu", "pb2_pair.cu", "pb2_energy64.cu", "pb2_bonded.cu",
                "pb2_integrate.cu", "pb2_nlist.cu", "pb2_noalloc.cu", "pb2_diag.cu",
                "pb2_transfer.cu", "pb2_minimize.cu", "pb2_pairlist.cu"]
CUDA_HEADERS = ["pb2_common.cuh", "pb2_divide.cuh", "pb2_kernels.cuh", "pb2_internal.h", "pb2_pairmath.cuh",
                "pb2_threefry.cuh", "pb2_obc_series.cuh", "pb2_bonded.cuh"]
HOST_SOURCES = ["synth_chain.c"]

# extra flags per source: the pair kernels flush subnormals and use the
# approximate divide (every value there is far from the subnormal range)
FILE_FLAGS = {"pb2_pair.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]}

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
  for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
    if cand and Path(cand).exists():
      return cand
  raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _stale(target: Path, sources) -> bool:
  if not target.exists():
    return True
  t = target.stat().st_mtime
  return any(s.exists() and s.stat().st_mtime > t for s in sources)


def build_host(force: bool = False) -> Path:
  srcs = [CSRC / s for s in HOST_SOURCES]
  if force or _stale(HOST_LIB, srcs):
    cc = shutil.which("gcc") or "cc"
    tmp = HOST_LIB.with_suffix(".so.tmp")
    subprocess.run([cc, "-O2", "-shared", "-fPIC", "-o", str(tmp), *map(str, srcs), "-lm"],
                   check=True)
    os.replace(tmp, HOST_LIB)
  return HOST_LIB


def build_cuda(force: bool = False, extra_flags=None) -> Path:
  present = [s for s in CUDA_SOURCES if (CSRC / s).exists()]
  srcs = [CSRC / s for s in present]
  deps = srcs + [CSRC / h for h in CUDA_HEADERS] + [INCLUDE / "prolix_b200.h"]
  if force or _stale(CUDA_LIB, deps):
    import concurrent.futures
    import tempfile
    nvcc = _nvcc()
    tmp = CUDA_LIB.with_suffix(".so.tmp")
    with tempfile.TemporaryDirectory() as td:
      objs = [Path(td) / (s.stem + ".o") for s in srcs]

      def compile_one(src_obj):
        src, obj = src_obj
        cmd = [nvcc, *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), *(extra_flags or []),
               "-I", str(INCLUDE), "-I", str(CSRC), "-c", "-o", str(obj), str(src)]
        return subprocess.run(cmd, capture_output=True, text=True)

      with concurrent.futures.ThreadPoolExecutor(max_workers=8) as ex:
        results = list(ex.map(compile_one, zip(srcs, objs)))
      for src, res in zip(srcs, results):
        if res.returncode != 0:
          raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stderr}")
      subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o",
                      str(tmp), *map(str, objs), "-lcuda"], check=True)
    os.replace(tmp, CUDA_LIB)
  return CUDA_LIB


FFI_SOURCE = CSRC / "ffi" / "pb2_ffi.cc"
FFI_LIB = PKG / "libprolix_b200_ffi.so"


def build_ffi(xla_include: str) -> Path:
  """The jax.ffi handler library, linked against libprolix_b200.so."""
  inc = Path(xla_include)
  if not (inc / "xla" / "ffi" / "api" / "ffi.h").exists():
    raise FileNotFoundError(f"{inc}/xla/ffi/api/ffi.h not found: XLA FFI headers are required")
  build_cuda()
  cuda_inc = Path(_nvcc()).resolve().parent.parent / "include"
  cxx = shutil.which("g++") or "c++"
  tmp = FFI_LIB.with_suffix(".so.tmp")
  subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(inc), "-I", str(INCLUDE),
                  "-I", str(cuda_inc), "-o", str(tmp), str(FFI_SOURCE), "-L", str(PKG),
                  "-lprolix_b200", f"-Wl,-rpath,{PKG}", "-L", str(cuda_inc.parent / "lib64"),
                  "-lcudart"], check=True)
  os.replace(tmp, FFI_LIB)
  return FFI_LIB


def build_all(force: bool = False) -> None:
  build_host(force)
  build_cuda(force)
  xla = os.environ.get("PB2_XLA_FFI_INCLUDE")
  if xla:
    build_ffi(xla)


if __name__ == "__main__":
  import argparse
  ap = argparse.ArgumentParser(description="build the prolix_b200 native libraries in-tree")
  ap.add_argument("--force", action="store_true")
  ap.add_argument("--ffi", metavar="XLA_INCLUDE", help="also build the jax.ffi handlers")
  args = ap.parse_args()
  build_all(args.force)
  if args.ffi:
    build_ffi(args.ffi)
