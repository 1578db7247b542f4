"""Restraints (sb_set_restraints) on the GPU against STORMM's own evaluation.

Fixture (tests/golden/make_golden.py --restraints-only): 40 constant restraints on a 60-atom
molecule, positional, distance, angle and dihedral, each kind with its measured value in every
region of the flat-bottom potential, with STORMM's energy of each, the total and the forces.
Restraints are evaluated in FP64: energies within 1e-9 relative plus half a unit of the energy
grid per restraint, forces within 1e-7 RMS relative.

Fixture (tests/golden/make_golden.py --ramps-only): 24 time-dependent restraints on the same
molecule (bounds, stiffnesses and targets ramped between two steps, or both steps equal), with
STORMM's energies and forces at steps before, at, within and after the ramps; same bounds."""
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


def _ramps(g, system=0, rows=None):
    out = []
    for row in (g["restraints"] if rows is None else rows):
        kind = int(row[0])
        v = row[7:]
        out.append({"system": system, "kind": kind, "atoms": [int(a) for a in row[1:1 + kind]],
                    "init_step": int(row[5]), "final_step": int(row[6]),
                    "k2": v[0], "k3": v[1], "r1": v[2], "r2": v[3], "r3": v[4], "r4": v[5],
                    "target": v[6:9], "final_k2": v[9], "final_k3": v[10], "final_r1": v[11],
                    "final_r2": v[12], "final_r3": v[13], "final_r4": v[14],
                    "final_target": v[15:18]})
    return out


@pytest.mark.parametrize("precision", [sb.PRECISION_SINGLE, sb.PRECISION_DOUBLE],
                         ids=["fp32", "fp64"])
def test_time_dependent_restraints_match_stormm(precision):
    g = load("restraint_ramps_r60.npz")
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol], precision=precision)
    _, f_plain = _restraint_only(syn, mol)
    n = len(g["restraints"])
    for step in g["steps"]:
        syn.set_restraints(_ramps(g))
        syn.set_restraint_step(int(step))
        e, f = _restraint_only(syn, mol)
        want = g["restraint_total_%d" % step][0]
        assert abs(e - want) <= 1e-9 * abs(want) + n * 2.0 ** -27, (step, e, want)
        frc = g["frc_restraint_%d" % step].reshape(-1, 3)
        if np.abs(frc).max() > 0.0:
            assert rms_rel(f - f_plain, frc) <= 1e-7, step
        else:
            assert np.array_equal(f, f_plain), step
        for q, row in enumerate(g["restraints"]):
            syn.set_restraints(_ramps(g, rows=[row]))
            eq, _ = _restraint_only(syn, mol)
            wq = g["restraint_energies_%d" % step][q]
            assert abs(eq - wq) <= 1e-9 * abs(wq) + 2.0 ** -26, (step, q, eq, wq)
    with pytest.raises(sb.StormmB200Error):
        syn.set_restraint_step(-1)
    bad = _ramps(g, rows=g["restraints"][:1])
    bad[0]["init_step"], bad[0]["final_step"] = 9, 3
    with pytest.raises(sb.StormmB200Error):
        syn.set_restraints(bad)
    syn.close()


def test_graph_minimizer_takes_the_cycle_count_as_the_step():
    """A positional target that moves during the minimization: the final energies take the
    restraint at the cycles run (an evaluation at that step on the final coordinates gives the
    same restraint energy to the bit), and the atom moves along the target's path."""
    g = load("restraints_r60.npz")
    mol = molecule_from_fixture(g)
    start = mol.coords[7] + 0.3
    end = mol.coords[7] + 1.5
    ramp = {"system": 0, "kind": sb.RESTRAINT_POSITION, "atoms": [7], "k2": 200.0, "k3": 200.0,
            "r1": 0.0, "r2": 0.0, "r3": 0.0, "r4": 5.0, "target": start, "init_step": 0,
            "final_step": 240, "final_k2": 200.0, "final_k3": 200.0, "final_r1": 0.0,
            "final_r2": 0.0, "final_r3": 0.0, "final_r4": 5.0, "final_target": end}
    syn = sb.Synthesis([mol])
    syn.set_restraints([ramp])
    syn.set_coordinates(mol.coords)
    cycles = 120
    syn.minimize(total_cycles=cycles, sd_cycles=30, convergence_rms=0.0, kernel=sb.MIN_GRAPH)
    slot = sb.NRG_SLOTS["restraint"]
    e_min = syn.energies_fixed()[0][slot]
    x = syn.coordinates()
    assert (x[7] - mol.coords[7]) @ (end - start) > 0.0
    syn.set_restraint_step(cycles)
    syn.set_coordinates(x)
    syn.initialize()
    syn.evaluate()
    assert syn.energies_fixed()[0][slot] == e_min
    syn.set_restraint_step(0)
    syn.initialize()
    syn.evaluate()
    assert syn.energies_fixed()[0][slot] != e_min
    syn.close()
