"""The FP64 oracle and the host topology against values computed by prolix's
own source code (``tests/golden/ref_fixtures.npz``, written by
``tests/golden/make_ref_fixtures.py``, which runs the reference's
force-field files unmodified on a NumPy stand-in for JAX).

This pins the oracle's restatement of the pair integral, the Born radii,
GB, ACE, Coulomb and LJ with the 1-4 table, bonds, angles, torsions,
periodic and harmonic impropers, Urey-Bradley, CMAP and the explicit 1-4
exception pairs to the reference itself, on synthetic chains and on the
charges and radii of a real protein (1A00 chain A).
"""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import ref_cases  # noqa: E402
from oracle import bonded as obonded  # noqa: E402
from oracle import energy as oenergy  # noqa: E402
from oracle import gbsa as ogbsa  # noqa: E402
from prolix_b200 import topology  # noqa: E402

FIX = np.load(ref_cases.FIXTURE)
TERMS = [str(t) for t in FIX["term_names"]]
E_REL = 1e-9
F_REL = 1e-8  # the finite-difference part of the fixture forces is good to ~1e-10


def oracle_system(name):
  """The case as the oracle takes it, with the reference's exclusion table."""
  s, cutoff = ref_cases.case_system(name)
  pairs, kind, lj14, c14 = topology.pairs_from_padded_table(
      FIX[f"{name}/excl_indices"], FIX[f"{name}/excl_scales_vdw"], FIX[f"{name}/excl_scales_elec"])
  s = dict(s, excl_pairs=pairs, excl_kind=kind)
  if f"{name}/exception_pairs" in FIX:
    p = FIX[f"{name}/exception_params"]
    s.update(exception_pairs=FIX[f"{name}/exception_pairs"], exception_chargeprods=p[:, 0],
             exception_sigmas=p[:, 1], exception_epsilons=p[:, 2])
  return s, cutoff, lj14, c14


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_inputs_are_rebuilt_identically(name):
  s, _ = ref_cases.case_system(name)
  assert str(FIX[f"{name}/input_digest"]) == ref_cases.digest(
      s["positions"], s["charges"], s["sigmas"], s["epsilons"], s["radii"], s["scaled_radii"])


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_finite_differences_agree_with_the_reference_backward_rule(name):
  assert float(FIX[f"{name}/fd_selfcheck"]) < 1e-8


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_oracle_energies_and_forces_match_the_reference(name):
  s, cutoff, lj14, c14 = oracle_system(name)
  e, f, ex = oenergy.energy_forces(s, s["positions"], cutoff, gb_cutoff=0.0, lj14=lj14, coul14=c14)
  ref = FIX[f"{name}/terms"]
  for i, t in enumerate(TERMS):
    got = e[t] if t != "total" else e["total"]
    assert got == pytest.approx(ref[i], rel=E_REL, abs=1e-9), t
  fr = FIX[f"{name}/forces"]
  assert np.linalg.norm(f - fr) / np.linalg.norm(fr) < F_REL
  np.testing.assert_allclose(ex["born_radii"], FIX[f"{name}/born_radii"], rtol=1e-12)


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_oracle_force_groups_match_the_reference(name):
  # LJ and Coulomb against the reference's analytic backward rules, the
  # bonded terms against differences of the reference energies
  s, cutoff, lj14, c14 = oracle_system(name)
  kw = dict(gb_cutoff=0.0, lj14=lj14, coul14=c14)
  f_all = ogbsa.nonbonded(s, s["positions"], cutoff, **kw)[1]
  f_no_lj = ogbsa.nonbonded(dict(s, epsilons=np.zeros_like(s["epsilons"])), s["positions"], cutoff,
                            **kw)[1]
  f_lj = f_all - f_no_lj
  ref_lj = FIX[f"{name}/forces_lj"]
  assert np.linalg.norm(f_lj - ref_lj) / np.linalg.norm(ref_lj) < 1e-10
  _, f_b = obonded.bonded_all(s, s["positions"])
  if "exception_pairs" in s:
    f_b = f_b + obonded.exception_pairs(s["positions"], s["exception_pairs"], s["exception_sigmas"],
                                        s["exception_epsilons"], s["exception_chargeprods"])[1]
  ref_b = FIX[f"{name}/forces_bonded"]
  assert np.linalg.norm(f_b - ref_b) / np.linalg.norm(ref_b) < F_REL


@pytest.mark.parametrize("name", [n for n in ref_cases.CASES if ref_cases.CASES[n][3]])
def test_cmap_coefficients_match_the_reference(name):
  s, _ = ref_cases.case_system(name)
  grids = np.asarray(s["cmap_energy_grids"], np.float64)
  ours = np.stack([topology.cmap_coefficients(g) for g in grids])
  ref = FIX[f"{name}/cmap_coeffs"]
  assert np.max(np.abs(ours - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
  oracle = np.stack([obonded.cmap_coefficients(g) for g in grids])
  assert np.max(np.abs(oracle - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("name", list(ref_cases.CASES))
def test_exclusion_table_matches_the_reference(name):
  # the pairs and classes the batch derives from the bonds equal the
  # reference's ExclusionSpec.from_protein + map_exclusions_to_dense_padded
  s, _ = ref_cases.case_system(name)
  n = len(s["charges"])
  pairs, kind, lj14, c14 = topology.pairs_from_padded_table(
      FIX[f"{name}/excl_indices"], FIX[f"{name}/excl_scales_vdw"], FIX[f"{name}/excl_scales_elec"])
  ours_p, ours_k = topology.exclusion_pairs(s["bonds"], n)
  if f"{name}/exception_pairs" in FIX:
    ours_k = np.zeros_like(ours_k)  # explicit 1-4 pairs are fully excluded (neighbor_list.py:117-119)
  else:
    assert lj14 == topology.LJ14_DEFAULT and c14 == topology.COUL14_DEFAULT
  np.testing.assert_array_equal(pairs, ours_p)
  np.testing.assert_array_equal(kind, ours_k)


def test_real_protein_born_radii_gb_and_ace_match_the_reference():
  c = ref_cases.PQR_CASE
  pos, q, rad, sr = (FIX[f"{c}/{k}"] for k in ("positions", "charges", "radii", "scaled_radii"))
  n = pos.shape[0]
  s = {"positions": pos, "charges": q, "radii": rad, "scaled_radii": sr, "sigmas": np.ones(n),
       "epsilons": np.zeros(n), "excl_pairs": np.zeros((0, 2), np.int32),
       "excl_kind": np.zeros(0, np.int32)}
  e, _, ex = ogbsa.nonbonded(s, pos, 0.0)
  np.testing.assert_allclose(ex["born_radii"], FIX[f"{c}/born_radii"], rtol=1e-12)
  assert e["gb"] == pytest.approx(float(FIX[f"{c}/gb"]), rel=E_REL)
  assert e["nonpolar"] == pytest.approx(float(FIX[f"{c}/nonpolar"]), rel=E_REL)


def test_padded_table_conversion_rejects_what_the_batch_cannot_hold():
  idx = np.array([[1, -1], [0, -1], [-1, -1]])
  ok = topology.pairs_from_padded_table(idx, np.zeros((3, 2)), np.zeros((3, 2)))
  np.testing.assert_array_equal(ok[0], [[0, 1]])
  with pytest.raises(ValueError, match="symmetric"):
    topology.pairs_from_padded_table(np.array([[1, -1], [-1, -1], [-1, -1]]), np.zeros((3, 2)),
                                     np.zeros((3, 2)))
  with pytest.raises(ValueError, match="twice"):
    topology.pairs_from_padded_table(np.array([[1, 1], [0, 0], [-1, -1]]), np.zeros((3, 2)),
                                     np.zeros((3, 2)))
  idx2 = np.array([[1, -1], [0, 2], [1, -1]])
  sv2 = np.array([[0.5, 1.0], [0.5, 0.4], [0.4, 1.0]])
  with pytest.raises(ValueError, match="one class"):
    topology.pairs_from_padded_table(idx2, sv2, np.full((3, 2), 0.8))


def test_nl_born_dense_gb_split_matches_the_reference():
  # prolix's compute_born_radii_neighbor_list and gb_energy_split_vjp
  # (generalized_born.py:266-337, :706-770), run from its own source with
  # every pair within the Born cutoff listed: the oracle's born_cutoff path
  c = ref_cases.SPLIT_CASE
  s, _ = ref_cases.case_system(ref_cases.SPLIT_BASE)
  r = np.asarray(s["positions"])
  assert str(FIX[f"{c}/input_digest"]) == ref_cases.digest(r, s["charges"], s["radii"], s["scaled_radii"])
  bc = float(FIX[f"{c}/born_cutoff"])
  assert bc == ref_cases.split_cutoff(r)
  # GB and ACE alone: no LJ (eps = 0), no direct Coulomb (k = 0)
  e, f, ex = ogbsa.nonbonded(dict(s, epsilons=np.zeros(len(r))), r, 0.0, k_coul=0.0, gb_cutoff=0.0,
                             born_cutoff=bc)
  np.testing.assert_allclose(ex["born_radii"], FIX[f"{c}/born_radii"], rtol=1e-12)
  assert e["gb"] == pytest.approx(float(FIX[f"{c}/gb"]), rel=E_REL)
  assert e["nonpolar"] == pytest.approx(float(FIX[f"{c}/nonpolar"]), rel=E_REL)
  fr = FIX[f"{c}/forces_gb_ace"]
  assert np.linalg.norm(f - fr) / np.linalg.norm(fr) < F_REL
