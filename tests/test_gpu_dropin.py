"""The prolix-facing Python API (make_energy_fn, nvt_langevin,
run_minimization, run_simulation) on the GPU, against the FP64 oracle."""

import types

import numpy as np
import pytest

from oracle import bonded as obonded
from oracle import gbsa as ogbsa
from oracle import integrator as ointeg
from oracle import prng
from prolix_b200 import engine, simulate, synth
from prolix_b200.system import exclusion_spec_from_bonds, make_energy_fn

pytestmark = pytest.mark.gpu


def oracle_terms(s, pos, cutoff, gb_cutoff):
  eb, fb = obonded.bonded_all(s, pos)
  en, fn, ex = ogbsa.nonbonded(s, pos, cutoff, gb_cutoff=gb_cutoff)
  e = {**eb, **en}
  e["total"] = sum(e.values())
  return e, fb + fn, ex


def spec_of(s):
  return exclusion_spec_from_bonds(s["bonds"], len(s["charges"]))


def test_make_energy_fn_default_semantics():
  # prolix: GB all pairs, LJ/Coulomb with cutoff_distance = 9.0
  s = synth.make_chain(400, 6, compact=True, cmap=True)
  fn = make_energy_fn(None, s, implicit_solvent=True, exclusion_spec=spec_of(s))
  e_ref, f_ref, _ = oracle_terms(s, s["positions"], 9.0, 0.0)
  assert fn(s["positions"]) == pytest.approx(e_ref["total"], rel=1e-6, abs=1e-6)
  f = fn.forces(s["positions"])
  assert np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref) < 1e-5
  terms = fn.terms(s["positions"])
  for k in ("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar"):
    assert terms[k] == pytest.approx(e_ref[k], rel=1e-6, abs=1e-6), k


def test_decomposed_dict_and_cutoff_keyword():
  s = synth.make_chain(200, 7, compact=True)
  d = make_energy_fn(None, s, implicit_solvent=True, return_decomposed=True, cutoff=0.0,
                     exclusion_spec=spec_of(s))
  assert set(d) == {"bond", "angle", "dihedral", "improper", "urey_bradley", "cmap", "lj",
                    "exception", "electrostatics", "nonpolar", "total"}
  e_ref, _, ex = oracle_terms(s, s["positions"], 0.0, 0.0)
  r = s["positions"]
  e_gb, e_coul, born = d["electrostatics"](r)
  assert e_gb == pytest.approx(e_ref["gb"], rel=1e-6)
  assert e_coul == pytest.approx(e_ref["coulomb"], rel=1e-6)
  np.testing.assert_allclose(born, ex["born_radii"], rtol=2e-6)
  assert d["lj"](r) == pytest.approx(e_ref["lj"], rel=1e-6, abs=1e-6)
  assert d["nonpolar"](r, born) == pytest.approx(e_ref["nonpolar"], rel=1e-6)
  assert d["total"](r) == pytest.approx(e_ref["total"], rel=1e-6)


def test_exclusion_spec_object():
  s = synth.make_chain(120, 9)
  from oracle import topology as otopo
  p12, p13, p14 = otopo.bonded_pairs(s["bonds"], 120)
  spec = types.SimpleNamespace(idx_12_13=np.concatenate([p12, p13]), idx_14=p14,
                               scale_14_elec=0.83333333, scale_14_vdw=0.5)
  fa = make_energy_fn(None, s, implicit_solvent=True, exclusion_spec=spec, cutoff=0.0)
  fb = make_energy_fn(None, s, implicit_solvent=True, exclusion_spec=spec_of(s), cutoff=0.0)
  assert fa(s["positions"]) == fb(s["positions"])
  e_ref = oracle_terms(s, s["positions"], 0.0, 0.0)[0]
  assert fa(s["positions"]) == pytest.approx(e_ref["total"], rel=1e-6)


def test_no_exclusion_information_excludes_nothing():
  # a dict without excl_indices and no exclusion_spec: the reference's
  # (N, 0) table (system.py:161-171), so 1-2 / 1-3 / 1-4 pairs interact fully
  s = synth.make_chain(120, 9)
  fn = make_energy_fn(None, s, implicit_solvent=True, cutoff=0.0)
  none = dict(s, excl_pairs=np.zeros((0, 2), np.int32), excl_kind=np.zeros(0, np.int32))
  e_ref, f_ref, _ = oracle_terms(none, s["positions"], 0.0, 0.0)
  t = fn.terms(s["positions"])
  for k in ("lj", "coulomb"):
    assert t[k] == pytest.approx(e_ref[k], rel=1e-6), k
  f = fn.forces(s["positions"])
  assert np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref) < 1e-5


def test_unknown_system_keys_raise():
  s = synth.make_chain(60, 3)
  with pytest.raises(ValueError, match="virtual_site_params"):
    make_energy_fn(None, dict(s, virtual_site_params=np.zeros((1, 12))), implicit_solvent=True)
  with pytest.raises(ValueError, match="atom_mask"):
    make_energy_fn(None, dict(s, atom_mask=np.arange(60) < 50), implicit_solvent=True)
  # metadata the reference's energy factory ignores too is accepted
  fn = make_energy_fn(None, dict(s, bond_mask=np.ones(59, bool), is_heavy=np.ones(60, bool)),
                      implicit_solvent=True)
  fn.close()


def test_separate_gb_and_direct_cutoffs():
  s = synth.make_chain(900, 10, compact=True)
  with engine.Batch([s], cutoff=8.0, gb_cutoff=12.0) as b:
    e, f = b.energy_forces()
    born = b.born_radii()
  e_ref, f_ref, ex = oracle_terms(s, s["positions"], 8.0, 12.0)
  assert np.linalg.norm(f - f_ref) / np.linalg.norm(f_ref) < 1e-5
  np.testing.assert_allclose(born, ex["born_radii"], rtol=2e-6)
  for i, k in enumerate(("bond", "angle", "dihedral", "cmap", "lj", "coulomb", "gb", "nonpolar")):
    assert e[0][i] == pytest.approx(e_ref[k], rel=1e-6, abs=1e-6), k


def test_nvt_langevin_protocol_matches_oracle():
  s = synth.make_chain(150, 11)
  fn = make_energy_fn(None, s, implicit_solvent=True, cutoff=0.0, exclusion_spec=spec_of(s))
  dt, kT, gamma = engine.akma_dt(1.0), 300 * engine.KB_KCAL, engine.akma_gamma(1.0)
  key = prng.prng_key(17)
  init_fn, apply_fn = simulate.nvt_langevin(fn, None, dt=dt, kT=kT, gamma=gamma, mass=s["masses"])
  st = init_fn(key, s["positions"], mass=s["masses"])
  for _ in range(3):
    st = apply_fn(st)
  force = lambda r: oracle_terms(s, r, 0.0, 0.0)[1]
  o = ointeg.init(force, key, s["positions"], s["masses"], kT, center=True)
  o = ointeg.run(o, force, 3, dt, kT, gamma)
  assert st.step == 3
  assert np.max(np.abs(st.position - o.position)) < 1e-7
  np.testing.assert_array_equal(st.rng, o.key)


def test_minimization_and_run_simulation():
  s = synth.make_chain(300, 12, compact=True)
  pos = s["positions"] + np.random.default_rng(0).normal(0, 0.15, size=s["positions"].shape)
  fn = make_energy_fn(None, dict(s, positions=pos), implicit_solvent=True, exclusion_spec=spec_of(s))
  e0 = fn(pos)
  r = simulate.run_minimization(fn, pos, sd_steps=30)
  assert fn(r) < e0
  out = simulate.run_simulation(s, pos, min_steps=10, therm_steps=20, key=prng.prng_key(2))
  assert out.shape == pos.shape and np.isfinite(out).all()


def test_device_pointer_entry_point_and_graph_capture():
  # pb2_energy_forces_device on torch device buffers equals the host entry
  # point, and replays inside a captured CUDA graph on new positions.
  import torch
  systems = [synth.make_chain(n, 60 + n, compact=True, cmap=True) for n in (166, 300)]
  with engine.Batch(systems) as b:
    e_host, f_host = b.energy_forces()
    n = b.n_atoms
    pos = torch.tensor(np.concatenate([s["positions"] for s in systems]), dtype=torch.float64,
                       device="cuda")
    e_dev = torch.zeros((2, e_host.shape[1]), dtype=torch.float64, device="cuda")
    f_dev = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    b.energy_forces_device(pos.data_ptr(), e_dev.data_ptr(), f_dev.data_ptr(), stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(f_dev.cpu().numpy(), f_host)
    np.testing.assert_array_equal(e_dev.cpu().numpy(), e_host)

    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
      b.energy_forces_device(pos.data_ptr(), e_dev.data_ptr(), f_dev.data_ptr(), side.cuda_stream)
    moved = pos.cpu().numpy() + 0.05 * np.sin(np.arange(3 * n)).reshape(n, 3)
    pos.copy_(torch.from_numpy(moved))
    g.replay()
    torch.cuda.synchronize()
    b.set_positions(moved)
    e_ref, f_ref = b.energy_forces()
    np.testing.assert_array_equal(f_dev.cpu().numpy(), f_ref)
    np.testing.assert_array_equal(e_dev.cpu().numpy(), e_ref)
    del g


def test_center_momentum_matches_the_oracle_init():
  # jax_md's center_velocity on each system of a ragged batch; a one-atom
  # system keeps its momentum
  keys = [prng.prng_key(k) for k in (3, 4, 5)]
  systems = [dict(synth.make_chain(n, n, compact=True), key=k) for n, k in zip((130, 1, 77), keys)]
  kT = 300 * engine.KB_KCAL
  with engine.Batch(systems, terms=0) as b:
    b.langevin_init()
    b.center_momentum()
    p = b.get_state(fields=("momentum",))["momentum"]
  zero = lambda r: np.zeros_like(r)
  for k, s in enumerate(systems):
    lo, hi = b.offsets[k], b.offsets[k + 1]
    o = ointeg.init(zero, keys[k], s["positions"], s["masses"], kT, center=True)
    np.testing.assert_allclose(p[lo:hi], o.momentum, rtol=0, atol=1e-13 * np.abs(o.momentum).max())
    if hi - lo > 1:
      assert np.abs(p[lo:hi].sum(axis=0)).max() < 1e-11 * np.abs(p[lo:hi]).max()
    else:
      np.testing.assert_array_equal(p[lo:hi], o.momentum)


def test_energy_fn_takes_cuda_arrays():
  # a CUDA tensor (or any DLPack producer on the device) is evaluated on the
  # device with no host copy; results equal the NumPy path bit for bit
  import torch
  s = synth.make_chain(180, 12, compact=True)
  fn = make_energy_fn(None, s, implicit_solvent=True, cutoff=0.0, exclusion_spec=spec_of(s))
  e_host, f_host = fn.energy_and_forces(s["positions"])
  t = torch.tensor(s["positions"], device="cuda")
  e_dev, f_dev = fn(t), fn.forces(t)
  assert e_dev.device.type == "cuda" and f_dev.device.type == "cuda" and tuple(f_dev.shape) == (180, 3)
  assert float(e_dev) == e_host
  np.testing.assert_array_equal(f_dev.cpu().numpy(), f_host)
  assert float(fn(torch.from_dlpack(t))) == e_host
  assert fn.terms(t)["total"] == e_host
  assert fn(torch.tensor(s["positions"])) == e_host  # CPU tensor: host path
  assert fn(s["positions"]) == e_host                # the host cache was dropped
  np.testing.assert_allclose(fn.born_radii(t), fn.born_radii(s["positions"]), rtol=0)
