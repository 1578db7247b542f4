"""The FP64-arithmetic mode (precision = SB_PRECISION_DOUBLE, STORMM's PrecisionModel::DOUBLE):
double parameters and double arithmetic, integer accumulation, every molecule tile by tile.

Against STORMM's FP64 CPU results the mode is limited only by its fixed-point grids, so these
tests raise the force and energy bits to 36 (2^-36 kcal/mol and kcal/mol/A) and hold energies
to 1e-10 of the summed terms and forces to 1e-10 RMS relative, four orders below the FP32
path's tolerances; the FP32 path is checked to sit between the two."""
import os

import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from stormm_b200 import synthetic
from fixtures import (load, molecule_from_fixture, reference_forces, reference_paths, rms_rel,
                      solvent_options)

pytestmark = pytest.mark.gpu

BITS = dict(frc_bits=36, nrg_bits=36)
CASES = ["synthetic_M0.npz", "synthetic_E2.npz", "synthetic_E17.npz", "synthetic_E33.npz",
         "synthetic_E257.npz", "synthetic_C600.npz", "synthetic_S64.npz", "synthetic_H100.npz",
         "synthetic_O100.npz", "synthetic_V100.npz", "synthetic_K64.npz", "synthetic_N7.npz",
         "synthetic_N8.npz"]


def _evaluate(g, precision, **extra):
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol], precision=precision, **solvent_options(g), **extra)
    syn.set_coordinates(mol.coords)
    syn.initialize()
    syn.evaluate()
    assert syn.status() == 0
    return syn


def _on_grid(xyz):
    """Coordinates as the synthesis holds them: rounded to its 2^-32 A fixed-point grid."""
    return np.round(np.asarray(xyz, dtype=np.float64) * 2.0 ** 32) / 2.0 ** 32


@pytest.mark.parametrize("name", CASES + [os.path.basename(p) for p in reference_paths()])
def test_fp64_mode_matches_stormm(name):
    """Energies against STORMM's FP64 sums; forces against the oracle (pinned to STORMM to
    1e-12) at the fixed-point coordinates, which the reference systems' coordinates are not on
    (their forces differ from STORMM's by the ~1e-10 A rounding alone)."""
    g = load(name)
    syn = _evaluate(g, sb.PRECISION_DOUBLE, **BITS)
    e = syn.energy_terms()[0]
    ref = g["energy_terms"]
    scale = max(np.abs(ref).sum(), 10.0)
    assert np.all(np.abs(e - ref) <= 1e-10 * scale), (e - ref)
    r = oracle.from_fixture(g).evaluate(_on_grid(g["coords"]))
    assert rms_rel(syn.forces(), r["forces"]) <= 1e-10
    if name.startswith("synthetic_"):
        # these fixtures were computed on the grid already
        assert rms_rel(syn.forces(), reference_forces(g)) <= 1e-10


@pytest.mark.parametrize("name", ["synthetic_M0.npz", "synthetic_C600.npz",
                                  "synthetic_S64.npz"])
def test_fp32_error_sits_between(name):
    """FP32 arithmetic loses several digits that the FP64 mode keeps."""
    g = load(name)
    ref_f = reference_forces(g)
    e64 = rms_rel(_evaluate(g, sb.PRECISION_DOUBLE, **BITS).forces(), ref_f)
    e32 = rms_rel(_evaluate(g, sb.PRECISION_SINGLE).forces(), ref_f)
    assert e64 * 1000.0 < e32 <= 5e-6, (e64, e32)


def test_fp64_mode_batches_repeat_and_match_alone():
    mols = [synthetic.make_molecule(synthetic._seed(6464, k), n, 0.2)
            for k, n in enumerate([12, 40, 77, 130, 33])]
    mols.append(synthetic.make_chain(6465, 900))
    xyz = np.concatenate([m.coords for m in mols])
    syn = sb.Synthesis(mols, precision=sb.PRECISION_DOUBLE, **BITS)
    syn.set_coordinates(xyz)
    syn.initialize()
    syn.evaluate()
    f1, e1 = syn.forces_fixed()[0].copy(), syn.energies_fixed().copy()
    syn.initialize()
    syn.evaluate()
    assert np.array_equal(syn.forces_fixed()[0], f1)
    assert np.array_equal(syn.energies_fixed(), e1)
    # the per-system launches give the same integers
    syn.initialize()
    syn.evaluate_range(0, len(mols))
    assert np.array_equal(syn.forces_fixed()[0], f1)
    assert np.array_equal(syn.energies_fixed(), e1)
    # and against the oracle, molecule by molecule
    f = syn.forces()
    off = 0
    for k, m in enumerate(mols):
        r = oracle.from_molecule(m).evaluate(_on_grid(m.coords))
        assert rms_rel(f[off:off + m.natom], r["forces"]) <= 1e-10, k
        scale = max(np.abs(r["energies"]).sum(), 10.0)
        assert np.all(np.abs(syn.energy_terms()[k] - r["energies"]) <= 1e-10 * scale), k
        off += m.natom


def test_fp64_mode_limits():
    mol = synthetic.make_molecule(5, 30, 0.1)
    syn = sb.Synthesis([mol], precision=sb.PRECISION_DOUBLE)
    syn.set_coordinates(mol.coords)
    with pytest.raises(sb.StormmB200Error, match="graph minimizer"):
        syn.minimize(total_cycles=3, kernel=sb.MIN_PERSISTENT)
    with pytest.raises(sb.StormmB200Error):
        sb.Synthesis([mol], precision=7)


def test_fp64_mode_clash_mitigated_evaluation_matches_stormm():
    """Softened Coulomb and Lennard-Jones cores (1-4 pairs included) in FP64 against STORMM's
    clash-mitigated FP64 evaluation of the same molecule, to the FP64 mode's tolerances."""
    g = load("synthetic_K64.npz")
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol], precision=sb.PRECISION_DOUBLE, **solvent_options(g), **BITS)
    syn.set_coordinates(mol.coords)
    syn.initialize()
    syn.evaluate_clash(float(g["clash_r0"][0]), float(g["clash_ratio"][0]))
    assert syn.status() == 0
    r = oracle.from_fixture(g).evaluate(_on_grid(mol.coords),
                                        clash_distance=float(g["clash_r0"][0]),
                                        clash_ratio=float(g["clash_ratio"][0]))
    scale = max(np.abs(r["energies"]).sum(), 10.0)
    assert np.all(np.abs(syn.energy_terms()[0] - r["energies"]) <= 1e-10 * scale)
    assert rms_rel(syn.forces(), r["forces"]) <= 1e-10
    # and against STORMM's own results at the unrounded coordinates, as the FP32 path
    scale = max(np.abs(g["clash_energy_terms"]).sum(), 10.0)
    assert np.all(np.abs(syn.energy_terms()[0] - g["clash_energy_terms"]) <= 1e-7 * scale)
    assert rms_rel(syn.forces(), g["clash_frc_total"].reshape(-1, 3)) <= 1e-7


@pytest.mark.parametrize("clash_cycles", [0, 4])
def test_fp64_mode_minimization_follows_the_oracle(clash_cycles):
    # wide softened cores (1 A, 0.9 sigma) so that the damped cycles change the trajectory
    soft = dict(clash_distance=1.0, clash_ratio=0.9)
    """STORMM's launchMinimization with PrecisionModel::DOUBLE: the graph minimizer over the
    FP64 evaluations with the conjugate direction kept in FP64, with and without clash-damped
    leading cycles.  Against the oracle's FP64
    minimizer (pinned to STORMM's CPU minimizer) from the same grid coordinates: the first ten
    cycles' energies to 1e-8 relative (1e-9 to 1e-10 measured) and the final energy within 1e-6
    of the energy drop (1e-9 to 1e-12 measured), and always closer than the FP32 path, which
    the minimization tests hold to 1e-5 over the first cycles and 1 % of the drop at the end.  What remains is the synthesis' 2^-32 A coordinate grid and 2^-36
    force grid, which the oracle does not round to: over many cycles a line-search comparison
    can still fall the other way."""
    mols = [synthetic.make_molecule(synthetic._seed(6161, k), n, 0.3)
            for k, n in enumerate([40, 64, 96])]
    cycles, sd = 60, 20
    syn = sb.Synthesis(mols, precision=sb.PRECISION_DOUBLE, **BITS)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    syn.minimize(total_cycles=cycles, sd_cycles=sd, clash_cycles=clash_cycles,
                 kernel=sb.MIN_GRAPH, record_history=True, **soft)
    assert syn.status() == 0
    hist = syn.minimize_history()
    f32 = sb.Synthesis(mols)
    f32.set_coordinates(np.concatenate([m.coords for m in mols]))
    f32.minimize(total_cycles=cycles, sd_cycles=sd, clash_cycles=clash_cycles,
                 kernel=sb.MIN_GRAPH, record_history=True, **soft)
    hist32 = f32.minimize_history()
    for k, m in enumerate(mols):
        _, h_ref = oracle.from_molecule(m).minimize(_on_grid(m.coords), cycles, sd,
                                                    clash_cycles=clash_cycles, **soft)
        rel64 = np.abs(hist[k] - h_ref) / np.abs(h_ref)
        rel32 = np.abs(hist32[k] - h_ref) / np.abs(h_ref)
        drop = h_ref[0] - h_ref[-1]
        print(f"molecule {k}: FP64 mode first-10 max rel {rel64[:10].max():.3e}, all "
              f"{rel64.max():.3e}, final / drop {abs(hist[k, -1] - h_ref[-1]) / drop:.3e}; "
              f"FP32 path all {rel32.max():.3e}, final / drop "
              f"{abs(hist32[k, -1] - h_ref[-1]) / drop:.3e}")
        assert rel64[:10].max() <= 1e-8, (k, rel64[:10].max())
        assert abs(hist[k, -1] - h_ref[-1]) <= 1e-6 * drop, k
        assert rel64.max() <= rel32.max(), k
