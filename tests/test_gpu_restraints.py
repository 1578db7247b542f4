"""Restraints (sb_set_restraints) on the GPU against STORMM's own evaluation.

Fixture (tests/golden/make_golden.py --restraints-only): 40 constant restraints on a 60-atom
molecule, positional, distance, angle and dihedral, each kind with its measured value in every
region of the flat-bottom potential, with STORMM's energy of each, the total and the forces.
Restraints are evaluated in FP64: energies within 1e-9 relative plus half a unit of the energy
grid per restraint, forces within 1e-7 RMS relative."""
import numpy as np
import pytest

import stormm_b200 as sb
from fixtures import load, molecule_from_fixture, rms_rel

pytestmark = pytest.mark.gpu


def _restraints(g, system=0, rows=None):
    out = []
    for row in (g["restraints"] if rows is None else rows):
        kind = int(row[0])
        out.append({"system": system, "kind": kind, "atoms": [int(v) for v in row[1:1 + kind]],
                    "k2": row[5], "k3": row[6], "r1": row[7], "r2": row[8], "r3": row[9],
                    "r4": row[10], "target": row[11:14]})
    return out


def _restraint_only(syn, mol, force=True):
    """Energy slot and forces of the restraints alone: a valence-only evaluation with them
    minus one without (the valence parts agree to the bit)."""
    syn.set_coordinates(mol.coords)
    syn.initialize()
    syn.evaluate(terms=sb.TERM_VALENCE)
    e = syn.energies()[0][sb.NRG_SLOTS["restraint"]]
    return e, syn.forces()


@pytest.mark.parametrize("precision", [sb.PRECISION_SINGLE, sb.PRECISION_DOUBLE],
                         ids=["fp32", "fp64"])
def test_restraints_match_stormm(precision):
    g = load("restraints_r60.npz")
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol], precision=precision)
    _, f_plain = _restraint_only(syn, mol)
    syn.set_restraints(_restraints(g))
    e, f = _restraint_only(syn, mol)
    n = len(g["restraints"])
    assert abs(e - g["restraint_total"][0]) <= 1e-9 * abs(g["restraint_total"][0]) + n * 2.0 ** -27
    assert rms_rel(f - f_plain, g["frc_restraint"].reshape(-1, 3)) <= 1e-7
    # one restraint at a time: every region of every kind
    for q, row in enumerate(g["restraints"]):
        syn.set_restraints(_restraints(g, rows=[row]))
        eq, _ = _restraint_only(syn, mol)
        assert abs(eq - g["restraint_energies"][q]) <= 1e-9 * abs(g["restraint_energies"][q]) + 2.0 ** -26, q
    syn.set_restraints([])
    e0, f0 = _restraint_only(syn, mol)
    assert e0 == 0.0 and np.array_equal(f0, f_plain)
    syn.close()


def test_restraints_per_system_and_minimization():
    """Restraints on the second of two copies only: the copies differ exactly by the
    restraints; per-system launches equal the batched one; the graph minimizer honours them
    (a strong positional restraint holds its atom) and the persistent kernel refuses them."""
    g = load("restraints_r60.npz")
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol, mol])
    syn.set_coordinates(np.concatenate([mol.coords, mol.coords]))
    syn.set_restraints(_restraints(g, system=1))
    syn.initialize()
    syn.evaluate()
    e = syn.energies()
    assert e[0][sb.NRG_SLOTS["restraint"]] == 0.0
    assert abs(e[1][sb.NRG_SLOTS["restraint"]] - g["restraint_total"][0]) < 1e-6
    batch = syn.energies_fixed()
    syn.initialize()
    syn.evaluate_range(0, 2)
    assert np.array_equal(syn.energies_fixed(), batch)
    with pytest.raises(sb.StormmB200Error, match="graph minimizer"):
        syn.minimize(total_cycles=10, kernel=sb.MIN_PERSISTENT)
    pin = {"system": 1, "kind": sb.RESTRAINT_POSITION, "atoms": [7], "k2": 500.0, "k3": 500.0,
           "r1": 0.0, "r2": 0.0, "r3": 0.0, "r4": 5.0, "target": mol.coords[7] + 0.5}
    syn.set_restraints([pin])
    syn.set_coordinates(np.concatenate([mol.coords, mol.coords]))
    syn.minimize(total_cycles=200, sd_cycles=50, kernel=sb.MIN_GRAPH)
    x = syn.coordinates()
    pulled = np.linalg.norm(x[mol.natom + 7] - (mol.coords[7] + 0.5))
    free = np.linalg.norm(x[7] - (mol.coords[7] + 0.5))
    assert pulled < 0.2 < free
    syn.close()
