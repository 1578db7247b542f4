"""The FP64 oracle against STORMM's own CPU evaluators and known answers.

Fixtures come from tests/golden/make_golden.py, which ran STORMM's CPU code
(Potential/valence_potential.tpp, Potential/nonbonded_potential.tpp) on the same inputs.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN

SYNTHETIC = sorted(glob.glob(os.path.join(GOLDEN, "synthetic_*.npz")))
REFERENCE = sorted(glob.glob(os.path.join(GOLDEN, "reference_*.npz")))


def _load(path):
    return dict(np.load(path))


def _total_force(g):
    return (g["frc_bond"] + g["frc_angle"] + g["frc_dihedral"] + g["frc_14"] +
            g["frc_nonbonded"] + g["frc_gb"]).reshape(-1, 3)


@pytest.mark.parametrize("path", SYNTHETIC + REFERENCE, ids=os.path.basename)
def test_energy_terms_match_stormm(path):
    g = _load(path)
    r = oracle.from_fixture(g).evaluate(g["coords"])
    ref = g["energy_terms"]
    np.testing.assert_allclose(r["energies"], ref, rtol=1e-10, atol=1e-9)


@pytest.mark.parametrize("path", SYNTHETIC + REFERENCE, ids=os.path.basename)
def test_forces_match_stormm(path):
    g = _load(path)
    r = oracle.from_fixture(g).evaluate(g["coords"])
    f = _total_force(g)
    rel = np.sqrt(((r["forces"] - f) ** 2).sum() / (f ** 2).sum())
    assert rel < 1e-12
    # the full MM driver (evalRestrainedMMGB) gives the same total force on the synthetic
    # molecules (which have no improper torsions)
    if "synthetic_" not in path:
        return
    ft = g["frc_total"].reshape(-1, 3)
    rel2 = np.sqrt(((r["forces"] - ft) ** 2).sum() / (ft ** 2).sum())
    assert rel2 < 1e-12


@pytest.mark.parametrize("path", SYNTHETIC + REFERENCE, ids=os.path.basename)
def test_gb_intermediates_match_stormm(path):
    g = _load(path)
    r = oracle.from_fixture(g).evaluate(g["coords"])
    np.testing.assert_allclose(r["psi"], g["gb_psi"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(r["radii"], g["gb_radii"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(r["sumdeijda"], g["gb_sumdeijda"], rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("path", REFERENCE, ids=os.path.basename)
def test_gb_known_answers(path):
    """GB energies asserted by test/Potential/test_generalized_born.cpp:296-330 (margin 1e-4)."""
    g = _load(path)
    r = oracle.from_fixture(g).evaluate(g["coords"], forces=False, terms=4)
    assert abs(r["energies"][8] - g["known_answer_gb"][0]) < 1e-4


def test_minimizer_reaches_reference_basin():
    """The oracle's restatement of the batched GPU line minimizer lowers the energy of the
    64-atom molecule into the same basin STORMM's CPU minimizer (a slightly different line
    search, MolecularMechanics/minimization.tpp) reaches after the same 100 cycles."""
    g = _load(os.path.join(GOLDEN, "synthetic_M0.npz"))
    m = _load(os.path.join(GOLDEN, "minimize_m0.npz"))
    s = oracle.from_fixture(g)
    _, hist = s.minimize(g["coords"], int(m["maxcyc"]), int(m["ncyc"]))
    ref_hist = m["min_potential_history"]
    assert abs(hist[0] - ref_hist[0]) < 1e-6 * abs(ref_hist[0])
    assert hist[-1] < hist[0]
    assert abs(hist[-1] - ref_hist[-1]) < 0.02 * abs(ref_hist[-1])


def test_split_fixed_point_conversions():
    """Numerics/accumulation.cui:126-160: values beyond the primary range spill whole units of
    2^31 (int63) or 2^63 (int95) into the overflow word."""
    assert oracle.float_to_int63(1234.5) == (1234, 0) or oracle.float_to_int63(1234.5) == (1235, 0)
    x, y = oracle.float_to_int63(3.0 * 2.0 ** 31 + 4096.0)
    assert y == 3 and x == 4096
    x, y = oracle.float_to_int63(-5.0 * 2.0 ** 31 - 2048.0)
    assert y == -5 and x == -2048
    x, y = oracle.double_to_int95(2.0 ** 64 + 2.0 ** 20)
    assert y == 2 and x == 2 ** 20


def test_clash_mitigated_evaluation_matches_stormm():
    """Softened Coulomb and Lennard-Jones cores (Potential/soft_core_potentials.tpp) as STORMM's
    MM driver applies them with a clash distance and a sigma ratio, 1-4 pairs included, on a
    molecule with close contacts: a few pairs below 1.5 A and many below 0.9 sigma."""
    g = _load(os.path.join(GOLDEN, "synthetic_K64.npz"))
    s = oracle.from_fixture(g)
    cd, cr = float(g["clash_r0"][0]), float(g["clash_ratio"][0])
    r = s.evaluate(g["coords"], clash_distance=cd, clash_ratio=cr)
    # STORMM's ScoreCard sums in fixed point at 2^-26 kcal/mol
    np.testing.assert_allclose(r["energies"], g["clash_energy_terms"], rtol=1e-9, atol=1e-5)
    ft = g["clash_frc_total"].reshape(-1, 3)
    assert np.sqrt(((r["forces"] - ft) ** 2).sum() / (ft ** 2).sum()) < 1e-12
    # the softened cores change the answer: the Lennard-Jones energy drops by orders of magnitude
    plain = s.evaluate(g["coords"])
    assert plain["energies"][4] > 1000.0 * r["energies"][4]
    np.testing.assert_allclose(plain["energies"], g["energy_terms_mm"], rtol=1e-9, atol=1e-5)


def test_clash_damped_minimization_reaches_reference_basin():
    """25 clash-damped cycles (cores shrinking linearly to nothing), then plain cycles: the same
    start energy as STORMM's CPU minimizer and the same basin after 60 cycles."""
    g = _load(os.path.join(GOLDEN, "synthetic_K64.npz"))
    m = _load(os.path.join(GOLDEN, "minimize_clash_k64.npz"))
    s = oracle.from_fixture(g)
    _, hist = s.minimize(g["coords"], int(m["maxcyc"]), int(m["ncyc"]),
                         clash_cycles=int(m["cdcyc"]), clash_distance=float(m["clash_r0"]),
                         clash_ratio=float(m["clash_ratio"]))
    ref_hist = m["min_potential_history"]
    assert abs(hist[0] - ref_hist[0]) < 1e-9 * abs(ref_hist[0])
    assert abs(hist[-1] - ref_hist[-1]) < 0.02 * abs(ref_hist[-1])


def test_oracle_matches_stormm_on_the_single_point_workload_sample():
    """The FP64 restatement against STORMM's own CPU build on 64 molecules of the 1,024-molecule
    workload (tests/golden/workload_single_point_sample.npz)."""
    from stormm_b200 import synthetic
    g = dict(np.load(os.path.join(GOLDEN, "workload_single_point_sample.npz")))
    mols = synthetic.workload_batched_single_point(1024, seed=synthetic.SEED_BASE + 1)
    offs = np.concatenate([[0], np.cumsum(g["natom"])])
    for j, k in enumerate(g["index"]):
        m = mols[k]
        c = g["coords"][offs[j]:offs[j + 1]]
        r = oracle.from_molecule(m).evaluate(c)
        np.testing.assert_allclose(r["energies"], g["energy_terms"][j], rtol=1e-11, atol=1e-10)
        f = g["forces"][offs[j]:offs[j + 1]]
        assert np.sqrt(((r["forces"] - f) ** 2).sum() / (f ** 2).sum()) < 1e-11


def _gpu_minimizer_case(case):
    """Molecules, starting coordinates and STORMM's launchMinimization histories of one case of
    tests/golden/gpu_minimize_<case>.npz (tests/golden/make_gpu_minimizer_golden.py)."""
    from stormm_b200 import synthetic
    g = _load(os.path.join(GOLDEN, f"gpu_minimize_{case}.npz"))
    start = g["start_coords"].reshape(-1, 3)
    mols, coords, off = [], [], 0
    for k, n in enumerate(g["sizes"]):
        mols.append(synthetic.make_molecule(synthetic._seed(int(g["seed"]), k), int(n),
                                            noise=float(g["noise"])))
        coords.append(start[off:off + n])
        off += n
    return g, mols, coords


@pytest.mark.parametrize("case", ["fp64", "fp64_clash"])
def test_minimizer_follows_stormm_gpu_minimizer(case):
    """The oracle's FP64 restatement of STORMM's GPU line minimizer against STORMM's own
    launchMinimization in PrecisionModel::DOUBLE on a B200 (12 molecules of 24-200 atoms, 200
    cycles, 50 steepest descent; with 25 clash-damped cycles in the second case): the same
    energy at the start of every one of the first 20 cycles to 1e-7 relative, while both take
    the same line-search decisions, and final energies within 1e-4 of the energy drop once
    rounding has steered the two runs apart."""
    g, mols, coords = _gpu_minimizer_case(case)
    cc = int(g["clash_cycles"])
    for k, (m, c0) in enumerate(zip(mols, coords)):
        _, h = oracle.from_molecule(m).minimize(c0, int(g["cycles"]), int(g["sd_cycles"]),
                                                clash_cycles=cc,
                                                clash_distance=float(g["clash_distance"]),
                                                clash_ratio=float(g["clash_ratio"]))
        s = g["history"][k]
        rel = np.abs(h[:21] - s[:21]) / np.maximum(np.abs(s[:21]), 1.0)
        assert rel.max() < 1e-7, (k, int(np.argmax(rel)), rel.max())
        drop = s[0] - s[-1]
        assert drop > 0 and abs(h[-1] - s[-1]) <= 1e-4 * drop, (k, h[-1], s[-1])
