"""The tiled path for large molecules (2,000-5,000-atom chains, or any molecule routed there by
tiled_above_atoms) against the fused path, STORMM's own results and the FP64 oracle.

The tiled path runs the fused kernel's valence code and pass-2 functor with the same integer
accumulation, but its GB passes differ in order: it sums psi over two pair streams per lane and
recomputes the HCT derivatives in pass 3, where the fused kernel walks one stream and stores the
derivatives from pass 1.  The two paths therefore agree to FP32 rounding (forces within 1e-6 RMS
relative and 2e-7 of the largest component, energies within 1e-7 of the summed terms), and each
is bit-identical from run to run.  Against FP64 the tolerances are those of the single-point
tests."""
import os

import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from stormm_b200 import synthetic
from fixtures import (FORCE_TOL, check_energies, fixture_magnitudes, load,
                      molecule_from_fixture, oracle_magnitudes, reference_forces, rms_rel)

pytestmark = pytest.mark.gpu



def _evaluate(mols, **opts):
    syn = sb.Synthesis(mols, **opts)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    syn.initialize()
    syn.evaluate()
    assert syn.status() == 0
    return syn


def _close(fused, tiled, rss):
    """The two FP32 paths sum in different orders: per-term bounds against each other."""
    e_f, e_t = fused.energy_terms(), tiled.energy_terms()
    for k in range(len(rss)):
        check_energies(e_t[k], e_f[k], rss[k], k)
    assert rms_rel(tiled.forces(), fused.forces()) <= 1e-6


def test_tiled_path_agrees_with_fused_and_repeats_exactly():
    mols = [synthetic.make_molecule(synthetic._seed(6060, k), n, 0.1)
            for k, n in enumerate([40, 100, 257, 300, 31])]
    mols.append(molecule_from_fixture(load("synthetic_C600.npz")))
    fused = _evaluate(mols)
    tiled = _evaluate(mols, tiled_above_atoms=32)
    rss = [oracle_magnitudes(m) for m in mols]
    _close(fused, tiled, rss)
    fp, _ = fused.forces_fixed()
    tp, _ = tiled.forces_fixed()
    assert np.abs(fp - tp).max() <= 2.0e-7 * np.abs(fp).max()
    for a, b in zip(fused.gb_workspace(), tiled.gb_workspace()):
        # psi summed in another order: the effective radii and the dE/dR sums (with their
        # cancellations) carry that FP32 rounding, so compare them as arrays
        assert rms_rel(b, a) <= 1e-6
        assert np.abs(b - a).max() <= 1e-6 * np.abs(a).max()
    prim, ovrf = tiled.forces_fixed()
    nrg = tiled.energies_fixed().copy()
    tiled.initialize()
    tiled.evaluate()
    assert np.array_equal(tiled.forces_fixed()[0], prim)
    assert np.array_equal(tiled.energies_fixed(), nrg)
    # energy-only and separate launchers as well
    for syn in (fused, tiled):
        syn.initialize()
        syn.evaluate(force=False, energy=True)
    e_f, e_t = fused.energy_terms(), tiled.energy_terms()
    for k in range(len(mols)):
        check_energies(e_t[k], e_f[k], rss[k], k)
    for syn in (fused, tiled):
        syn.initialize()
        syn.launch_valence()
        syn.launch_nonbonded()
    _close(fused, tiled, rss)


def test_tiled_chain_fixture_matches_stormm():
    g = load("synthetic_C600.npz")
    syn = _evaluate([molecule_from_fixture(g)], tiled_above_atoms=256)
    check_energies(syn.energy_terms()[0], g["energy_terms"], fixture_magnitudes(g))
    assert rms_rel(syn.forces(), reference_forces(g)) <= FORCE_TOL


def test_large_chains_against_oracle():
    mols = [synthetic.make_chain(synthetic._seed(7070, k), n) for k, n in enumerate([2100, 2700])]
    syn = _evaluate(mols)
    energies = syn.energy_terms()
    forces = syn.split(syn.forces())
    for k, m in enumerate(mols):
        ref = oracle.from_molecule(m).evaluate(m.coords)
        check_energies(energies[k], ref["energies"], oracle_magnitudes(m), k)
        assert rms_rel(forces[k], ref["forces"]) <= FORCE_TOL, k


def test_tiled_per_system_launches_equal_batched_and_persistent_minimization_is_rejected():
    mols = [synthetic.make_chain(synthetic._seed(7171, 0), 2200),
            synthetic.make_molecule(synthetic._seed(7171, 1), 90, 0.1),
            synthetic.make_chain(synthetic._seed(7171, 2), 2050)]
    syn = _evaluate(mols)
    f_b = syn.forces_fixed()
    e_b = syn.energies_fixed().copy()
    syn.initialize()
    syn.evaluate_range(0, len(mols))
    assert np.array_equal(syn.forces_fixed()[0], f_b[0])
    assert np.array_equal(syn.energies_fixed(), e_b)
    with pytest.raises(sb.StormmB200Error, match="graph minimizer"):
        syn.minimize(total_cycles=2, kernel=sb.MIN_PERSISTENT)


def _graph_minimize(mols, cycles, **opts):
    syn = sb.Synthesis(mols, **opts)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    syn.minimize(total_cycles=cycles, sd_cycles=10, clash_cycles=4, kernel=sb.MIN_GRAPH,
                 record_history=True)
    assert syn.status() == 0
    return syn


def test_graph_minimization_of_tiled_molecules_follows_the_oracle():
    """Molecules on the tiled path minimize with the graph minimizer: the tiled evaluations take
    the place of the fused ones in each cycle's graph.  Small molecules routed there
    (tiled_above_atoms=32) follow the FP64 oracle's minimizer as the fused path does: the first
    trial energies to 1e-5 relative, the final energy within 1 % of the drop."""
    mols = [synthetic.make_molecule(synthetic._seed(7272, k), n, 0.3)
            for k, n in enumerate([40, 64, 96])]
    cycles = 40
    syn = _graph_minimize(mols, cycles, tiled_above_atoms=32)
    hist = syn.minimize_history()
    for k, m in enumerate(mols):
        _, h_ref = oracle.from_molecule(m).minimize(m.coords, cycles, 10, clash_cycles=4)
        np.testing.assert_allclose(hist[k, :3], h_ref[:3], rtol=1e-5, err_msg=f"molecule {k}")
        drop = h_ref[0] - h_ref[-1]
        assert abs(hist[k, -1] - h_ref[-1]) <= 0.01 * drop + 1e-3, (k, hist[k, -1], h_ref[-1])


def test_graph_minimization_mixes_tiled_and_fused_molecules():
    """A 2,200-atom chain beside small molecules: the small ones minimize exactly as without
    the chain, the chain exactly as alone and as in the per-system launch sequence, and its
    energy falls."""
    chain = synthetic.make_chain(synthetic._seed(7373, 0), 2200, 0.2)
    small = [synthetic.make_molecule(synthetic._seed(7373, k), n, 0.3)
             for k, n in enumerate([30, 75, 120], start=1)]
    cycles = 25
    mixed = _graph_minimize(small + [chain], cycles)
    only_small = _graph_minimize(small, cycles)
    alone = _graph_minimize([chain], cycles)
    n_small = sum(m.natom for m in small)
    assert np.array_equal(mixed.coordinates()[:n_small], only_small.coordinates())
    assert np.array_equal(mixed.energies_fixed()[:3], only_small.energies_fixed())
    assert np.array_equal(mixed.coordinates()[n_small:], alone.coordinates())
    assert np.array_equal(mixed.energies_fixed()[3], alone.energies_fixed()[0])
    h = mixed.minimize_history()[3]
    assert h[-1] < h[0]
    per_system = sb.Synthesis([chain])
    per_system.set_coordinates(chain.coords)
    per_system.minimize_range(0, 1, total_cycles=cycles, sd_cycles=10, clash_cycles=4,
                              kernel=sb.MIN_GRAPH)
    assert np.array_equal(per_system.coordinates(), alone.coordinates())
