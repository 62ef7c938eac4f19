"""Host-side logic and the C ABI library surface (no GPU calls)."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import bonded as obonded
from oracle import topology as otopo
from prolix_b200 import _build, _lib, engine, synth, topology

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
  text = (ROOT / "include" / "prolix_b200.h").read_text()
  return sorted(set(re.findall(r"\b(pb2_[a-z_0-9]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
  lib = _lib.load()
  declared = header_symbols()
  assert len(declared) >= 20
  for name in declared:
    assert hasattr(lib, name), name
  bound = {name for name, _, _ in _lib.SIGNATURES}
  assert set(declared) <= bound | {"pb2_ctx_create"}
  assert lib.pb2_abi_version() == _lib.ABI_VERSION == 3


def _struct_fields(text, name):
  body = text[text.index("typedef struct " + name):text.index("} " + name + ";")]
  body = body[body.index("{") + 1:]
  body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
  out = []
  for decl in body.split(";"):
    decl = decl.strip()
    if not decl:
      continue
    head, *rest = decl.split(",")
    names = [head.split()[-1]] + [r.strip() for r in rest]
    out.extend(n.lstrip("*").split("[")[0] for n in names)
  return out


def test_ctypes_struct_layout_matches_header():
  text = (ROOT / "include" / "prolix_b200.h").read_text()
  assert _struct_fields(text, "pb2_system_desc") == [f[0] for f in _lib.SystemDesc._fields_]
  assert _struct_fields(text, "pb2_run_params") == [f[0] for f in _lib.RunParams._fields_]


def test_no_device_reports_enodev():
  lib = _lib.load()
  h = ctypes.c_void_p()
  try:
    import torch
    has_gpu = torch.cuda.is_available()
  except Exception:
    has_gpu = False
  if has_gpu:
    pytest.skip("a GPU is present")
  assert lib.pb2_ctx_create(0, ctypes.byref(h)) == -7


def test_synth_is_seed_deterministic():
  a = synth.make_chain(300, 17, compact=True, cmap=True)
  b = synth.make_chain(300, 17, compact=True, cmap=True)
  for k in a:
    np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]))
  c = synth.make_chain(300, 18, compact=True)
  assert not np.array_equal(a["positions"], c["positions"])
  assert abs(a["charges"].sum()) < 1e-12


def test_synth_distributions_and_geometry():
  s = synth.make_chain(2500, 3, compact=True)
  n = 2500
  assert s["positions"].shape == (n, 3)
  assert (s["sigmas"] >= 1.0).all() and (s["sigmas"] <= 3.4).all()
  assert (s["epsilons"] >= 0.01).all() and (s["epsilons"] <= 0.2).all()
  assert (s["radii"] >= 1.2).all() and (s["radii"] <= 1.9).all()
  sf = s["scaled_radii"] / s["radii"]
  assert (sf >= 0.72).all() and (sf <= 0.85).all()
  d = np.linalg.norm(np.diff(s["positions"], axis=0), axis=1)
  np.testing.assert_allclose(d, s["bond_params"][:, 0], rtol=1e-9)
  assert (d >= 1.0).all() and (d <= 1.53).all()
  r = np.linalg.norm(s["positions"], axis=1)
  assert r.max() < 1.5 * synth.globule_radius(n)
  from scipy.spatial import cKDTree
  pairs = cKDTree(s["positions"]).query_pairs(2.5, output_type="ndarray")
  assert np.all(np.abs(pairs[:, 0] - pairs[:, 1]) < 3)


def test_batch_sizes_log_uniform():
  sizes = synth.batch_sizes(512, 2024)
  assert sizes.min() >= 150 and sizes.max() <= 4000
  assert 900 < sizes.mean() < 1500


def test_exclusions_match_oracle_rule():
  s = synth.make_chain(80, 2)
  pairs, kind = topology.exclusion_pairs(s["bonds"], 80)
  p12, p13, p14 = otopo.bonded_pairs(s["bonds"], 80)
  assert len(pairs) == len(p12) + len(p13) + len(p14)
  assert (kind == 1).sum() == len(p14)


def test_cmap_coefficients_match_oracle():
  g = np.random.default_rng(9).uniform(-2, 2, size=(24, 24))
  np.testing.assert_allclose(topology.cmap_coefficients(g), obonded.cmap_coefficients(g),
                             atol=1e-12)


def test_prepare_system_defaults_and_units():
  s = synth.make_chain(40, 1)
  p = engine.prepare_system(s)
  assert p["dt"] == pytest.approx(1.0 / 48.88821291839)
  assert p["kT"] == pytest.approx(300 * 0.0019872041)
  assert p["gamma"] == pytest.approx(1.0 * 48.88821291839e-3)
  assert p["excl_pairs"].dtype == np.int32 and (p["excl_pairs"][:, 0] < p["excl_pairs"][:, 1]).all()
  d = engine._desc(p)
  assert d.n_atoms == 40 and d.n_bonds == 39 and d.n_torsion_terms == 1


def test_build_flags_target_sm100a_only():
  flags = " ".join(_build.NVCC_FLAGS)
  assert "arch=compute_100a,code=sm_100a" in flags
  assert "sm_90" not in flags


def test_far_field_polynomials_meet_float32_bound():
  # The pair kernels evaluate the OBC far-field series V(u) (descreening) and
  # D(u) (chain rule) by the tier polynomials of pb2_obc_series.cuh, on tiles
  # whose smallest box separation keeps u = (s/r)^2 below the tier's bound
  # (pb2_api.cu tier2, pb2_pair.cu tile2_kernel).  With the float32
  # coefficients the kernels use, the relative error against the full series
  # must stay below half a float32 ulp in exact arithmetic, and below one ulp
  # when evaluated by float32 Horner steps.
  txt = (ROOT / "prolix_b200" / "csrc" / "pb2_obc_series.cuh").read_text()

  def exact(u, der):
    k = np.arange(1, 301, dtype=np.float64)[:, None]
    c = 2.0 * k * (k + 1) / (2 * k + 1) if der else k / (2 * k + 1)
    return (c * u[None, :] ** (k - 1)).sum(0)

  bounds = {}
  for name, der in (("Value", False), ("Deriv", True)):
    us = re.search(r"k%sTierU\[4\] = \{([^}]*)\}" % name, txt).group(1)
    bounds[der] = [float(v) for v in us.split(",")]
  assert bounds[False][3] == bounds[True][3] == 0.16  # the near-tile per-pair test bound
  n_poly = 0
  for m in re.finditer(r"struct ObcPoly<(true|false), (\d)> \{(.*?)\n\};", txt, re.S):
    der, tier = m.group(1) == "true", int(m.group(2))
    coef = [float(v) for v in re.findall(r"make_float2\(([-0-9.e+]+)f,", m.group(3))]
    assert coef and all(np.float32(c) == c for c in coef)
    u = np.linspace(0.0, bounds[der][tier], 20001)
    ref = exact(u, der)
    p64 = np.zeros_like(u)
    p32 = np.zeros_like(u, dtype=np.float32)
    u32 = u.astype(np.float32)
    for c in coef:  # highest power first
      p64 = p64 * u + c
      p32 = (p32.astype(np.float64) * u32 + c).astype(np.float32)  # one rounding per step, as fma
    assert np.max(np.abs(p64 - ref) / ref) < 6e-8, (der, tier)
    assert np.max(np.abs(p32 - ref) / ref) < 1.2e-7, (der, tier)
    n_poly += 1
  assert n_poly == 8


def test_exclusion_pairs_match_breadth_first_search():
  # 1-2 / 1-3 / 1-4 classes by shortest bond separation (prolix
  # utils/topology.py:26-93) on chains, branched trees, rings and a
  # multi-bond topology, against an independent breadth-first search.
  from collections import deque

  from prolix_b200 import topology

  def bfs_classes(bonds, n):
    adj = [[] for _ in range(n)]
    for i, j in bonds:
      if i != j:
        adj[i].append(j)
        adj[j].append(i)
    out = {}
    for s in range(n):
      dist = {s: 0}
      q = deque([s])
      while q:
        u = q.popleft()
        if dist[u] == 3:
          continue
        for v in adj[u]:
          if v not in dist:
            dist[v] = dist[u] + 1
            q.append(v)
      for t, d in dist.items():
        if t > s and d >= 1:
          out[(s, t)] = 0 if d <= 2 else 1
    return out

  rng = np.random.default_rng(5)
  cases = [np.stack([np.arange(30), np.arange(1, 31)], 1),                     # chain
           np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 5], [5, 0], [2, 6]]),  # ring + branch
           np.array([[0, 1], [0, 2], [0, 3], [0, 4], [4, 5], [5, 6], [1, 1]])]  # star, self bond
  for _ in range(5):  # random trees with extra ring-closing bonds
    n = 60
    par = np.array([rng.integers(0, k) for k in range(1, n)])
    b = np.stack([par, np.arange(1, n)], 1)
    extra = rng.integers(0, n, size=(4, 2))
    cases.append(np.concatenate([b, extra, b[:3]]))
  for b in cases:
    n = int(b.max()) + 1
    pairs, kind = topology.exclusion_pairs(b, n)
    got = {(int(i), int(j)): int(k) for (i, j), k in zip(pairs, kind)}
    assert got == bfs_classes(b.tolist(), n)
    assert np.all(pairs[:, 0] < pairs[:, 1])


def test_exclusion_finder_rejects_bad_bond_indices():
  import pytest

  from prolix_b200 import topology
  with pytest.raises(ValueError, match="out of range"):
    topology.exclusion_pairs(np.array([[0, 1], [2, 5]]), 5)
  with pytest.raises(ValueError, match="out of range"):
    topology.exclusion_pairs(np.array([[-1, 1]]), 5)


def test_streamed_partition_covers_systems_in_balanced_ranges():
  from prolix_b200 import streamed
  rng = np.random.default_rng(5)
  sizes = np.exp(rng.uniform(np.log(150), np.log(4000), 512)).astype(int)
  r = streamed.partition(sizes, 4)
  assert r[0][0] == 0 and r[-1][1] == len(sizes)
  assert all(a < b for a, b in r) and all(r[g][1] == r[g + 1][0] for g in range(len(r) - 1))
  work = [float(np.sum(sizes[a:b].astype(float) ** 2)) for a, b in r]
  assert max(work) / min(work) < 1.2
  assert streamed.partition([10, 20], 5) == [(0, 1), (1, 2)]
  assert streamed.partition([10], 3) == [(0, 1)]


def test_bench_reads_the_kernels_series_tiers():
  # bench.py's flop counts follow the tier table the kernels compile
  import bench
  tiers = bench.series_tiers()
  assert tiers["value"] == ([0.0075, 0.036, 0.089, 0.16], [3, 4, 5, 6])
  assert tiers["deriv"] == ([0.027, 0.07, 0.129, 0.16], [4, 5, 6, 7])
  systems = synth.make_batch(4, 11, 150, 600, compact=True, **synth.PHYSICAL_RANGES)
  k = bench.series_terms(systems)
  assert 3.0 <= k["value"] <= 6.0 and 4.0 <= k["deriv"] <= 7.0
  f = bench.flops_per_pair(k)
  assert f["born"] == 4 * k["value"] + 14 and f["chain"] == 4 * k["deriv"] + 27 and f["force"] == 55.0


def test_prepare_system_packs_exception_pairs():
  # ExclusionSpec field names -> descriptor (pairs, (charge product, sigma, epsilon))
  s = synth.make_chain(30, 2)
  ex = dict(s, exception_pairs=np.array([[0, 3], [5, 8]]), exception_chargeprods=[0.1, -0.2],
            exception_sigmas=[3.0, 3.1], exception_epsilons=[0.05, 0.07])
  p = engine.prepare_system(ex)
  assert p["exception_pairs"].dtype == np.int32 and p["exception_pairs"].shape == (2, 2)
  np.testing.assert_array_equal(p["exception_params"], [[0.1, 3.0, 0.05], [-0.2, 3.1, 0.07]])
  d = engine._desc(p)
  assert d.n_exceptions == 2
  q = engine.prepare_system(s)
  assert q["exception_pairs"].shape == (0, 2) and engine._desc(q).n_exceptions == 0


def test_ffi_handlers_are_source_behind_a_build_flag():
  # the jax.ffi handlers exist as source; building them needs XLA's headers,
  # which this image lacks, and the default build leaves them out
  src = ROOT / "prolix_b200" / "csrc" / "ffi" / "pb2_ffi.cc"
  text = src.read_text()
  for name in ("pb2_ffi_energy_forces", "pb2_ffi_baoab", "pb2_energy_forces_device",
               "pb2_langevin_run_device"):
    assert name in text
  with pytest.raises(FileNotFoundError, match="XLA FFI headers"):
    _build.build_ffi(str(ROOT / "no_such_xla_include"))
