"""CUDA path against the FP64 oracle and STORMM's own CPU results, through the C ABI.

Tolerances (FP32 arithmetic with fixed-point accumulation against FP64), as tests/fixtures.py
states them:
* energies: each term within 1e-6 of the largest of |E_term|, 1 kcal/mol and the root-sum-square
  of the term's contributions;
* forces: RMS relative error at most 5e-6 against FP64;
* fixed-point sums: bit-identical across runs, across batch compositions and between the batched
  and the per-system launches.
"""
import os

import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from fixtures import (FORCE_TOL, check_energies, default_solvent_paths, fixture_magnitudes,
                      load, molecule_from_fixture, oracle_magnitudes, reference_forces,
                      reference_paths, rms_rel, solvent_options, synthetic_paths)

pytestmark = pytest.mark.gpu


def _run(mols, igb=5, dielectric=80.0, terms=sb.TERM_ALL, coords=None, **opts):
    syn = sb.Synthesis(mols, igb=igb, dielectric=dielectric, **opts)
    xyz = np.concatenate([m.coords for m in mols]) if coords is None else coords
    syn.set_coordinates(xyz)
    syn.initialize()
    syn.evaluate(terms=terms)
    out = {"energies": syn.energy_terms(), "forces": syn.forces(), "syn": syn}
    assert syn.status() == 0
    return out


@pytest.mark.parametrize("path", synthetic_paths(), ids=os.path.basename)
def test_single_system_matches_stormm(path):
    g = load(os.path.basename(path))
    mol = molecule_from_fixture(g)
    r = _run([mol], **solvent_options(g))
    check_energies(r["energies"][0], g["energy_terms"], fixture_magnitudes(g), path)
    err = rms_rel(r["forces"], reference_forces(g))
    assert err <= FORCE_TOL, err


@pytest.mark.parametrize("path", reference_paths(), ids=os.path.basename)
def test_reference_systems_known_answers(path):
    """Trp-cage and alanine dipeptide under HCT, OBC, OBC-II and the two neck models, against
    STORMM's CPU results and the known GB energies of
    test/Potential/test_generalized_born.cpp:296-300."""
    g = load(os.path.basename(path))
    mol = molecule_from_fixture(g)
    r = _run([mol], **solvent_options(g))
    check_energies(r["energies"][0], g["energy_terms"], fixture_magnitudes(g), path)
    assert abs(r["energies"][0][8] - g["known_answer_gb"][0]) < 1e-3
    assert rms_rel(r["forces"], reference_forces(g)) <= FORCE_TOL


def test_gb_workspace_matches_stormm():
    g = load("synthetic_E100.npz")
    r = _run([molecule_from_fixture(g)])
    psi, rad, sde = r["syn"].gb_workspace()
    np.testing.assert_allclose(psi, g["gb_psi"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(rad, g["gb_radii"], rtol=1e-5)
    np.testing.assert_allclose(sde, g["gb_sumdeijda"], rtol=1e-4, atol=1e-4)


def test_batch_of_mixed_sizes_is_bit_identical_to_single_runs():
    paths = default_solvent_paths()
    mols = [molecule_from_fixture(load(os.path.basename(p))) for p in paths]
    batch = _run(mols)
    prim_b, ovrf_b = batch["syn"].forces_fixed()
    ef_b = batch["syn"].energies_fixed()
    offs = []
    for k, m in enumerate(mols):
        single = _run([m])
        prim_s, ovrf_s = single["syn"].forces_fixed()
        _, off = _system_layout(batch["syn"], k)
        n = m.natom
        assert np.array_equal(prim_b[:, off:off + n], prim_s[:, :n])
        assert np.array_equal(ovrf_b[:, off:off + n], ovrf_s[:, :n])
        assert np.array_equal(ef_b[k], single["syn"].energies_fixed()[0])
        offs.append(off)
    # and each system still matches STORMM
    for k, p in enumerate(paths):
        g = load(os.path.basename(p))
        check_energies(batch["energies"][k], g["energy_terms"], fixture_magnitudes(g), p)


def _system_layout(syn, k):
    import ctypes
    n, off = ctypes.c_int(), ctypes.c_int()
    sb.library().sb_system_atoms(syn.handle, k, ctypes.byref(n), ctypes.byref(off))
    return n.value, off.value


def test_run_to_run_bit_identical():
    mols = [molecule_from_fixture(load("synthetic_E300.npz")),
            molecule_from_fixture(load("synthetic_M0.npz"))]
    a = _run(mols)["syn"]
    first = a.forces_fixed()
    first_e = a.energies_fixed()
    for _ in range(3):
        a.initialize()
        a.evaluate()
        again = a.forces_fixed()
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[1], again[1])
        assert np.array_equal(first_e, a.energies_fixed())


def test_block_size_changes_no_bit():
    """A launch of few work units runs 512-thread blocks; 256 threads (set explicitly) give the
    same fixed-point forces and energies, force+energy and energy-only."""
    mols = [molecule_from_fixture(load(os.path.basename(p))) for p in default_solvent_paths()]
    wide = _run(mols)["syn"]
    narrow = _run(mols, threads_per_block=256)["syn"]
    units = wide.launch_info()["work_units"]
    assert units < 4 * 148
    for syn in (wide, narrow):
        syn.initialize()
        syn.evaluate()
    a, b = wide.forces_fixed(), narrow.forces_fixed()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(wide.energies_fixed(), narrow.energies_fixed())
    for syn in (wide, narrow):
        syn.initialize()
        syn.evaluate(force=False)
    assert np.array_equal(wide.energies_fixed(), narrow.energies_fixed())
    wide.close()
    narrow.close()


def test_asynchronous_download_matches_the_getters():
    """Two syntheses on two streams, results read back with sb_download_results_async into
    page-locked buffers: equal to the synchronous getters; pageable buffers are refused."""
    import torch
    mols = [molecule_from_fixture(load(os.path.basename(p))) for p in default_solvent_paths()]
    syns = [sb.Synthesis(mols), sb.Synthesis(mols)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    xyz = np.concatenate([m.coords for m in mols])
    n = xyz.size
    pf = [torch.zeros(n, dtype=torch.float64).pin_memory().numpy() for _ in range(2)]
    pe = [torch.zeros(len(mols) * sb.NRG_STRIDE, dtype=torch.float64).pin_memory().numpy()
          for _ in range(2)]
    for b in range(2):
        h = streams[b].cuda_stream
        syns[b].set_coordinates(xyz, stream=h)
        syns[b].initialize(stream=h)
        syns[b].evaluate(stream=h)
        syns[b].download_async(pf[b], pe[b], stream=h)
    torch.cuda.synchronize()
    for b in range(2):
        np.testing.assert_array_equal(pf[b], syns[b].forces().reshape(-1))
        np.testing.assert_array_equal(pe[b], syns[b].energies().reshape(-1))
    with pytest.raises(sb.StormmB200Error, match="page-locked"):
        syns[0].download_async(np.zeros(n), None)
    for s in syns:
        s.close()


def test_per_system_launches_match_batched():
    mols = [molecule_from_fixture(load(os.path.basename(p)))
            for p in default_solvent_paths()[:6]]
    batch = _run(mols)["syn"]
    ref_prim, ref_ovrf = batch.forces_fixed()
    ref_e = batch.energies_fixed()
    batch.initialize()
    batch.evaluate_range(0, len(mols))
    prim, ovrf = batch.forces_fixed()
    assert np.array_equal(prim, ref_prim) and np.array_equal(ovrf, ref_ovrf)
    assert np.array_equal(batch.energies_fixed(), ref_e)


def test_separate_launchers_sum_to_fused():
    """launchNonbonded followed by launchValence equals the fused pass.  Different kernel
    variants may round an FP32 partial sum differently, so the comparison is to FP32 rounding,
    not to the bit."""
    mols = [molecule_from_fixture(load("synthetic_M0.npz")),
            molecule_from_fixture(load("synthetic_E48.npz"))]
    syn = _run(mols)["syn"]
    fused_e = syn.energy_terms()
    fused_f = syn.forces()
    syn.initialize()
    syn.launch_nonbonded()
    syn.launch_valence()
    for k in range(len(mols)):
        check_energies(syn.energy_terms()[k], fused_e[k], oracle_magnitudes(mols[k]))
    assert rms_rel(syn.forces(), fused_f) < 1e-6


def test_energy_only_matches_force_energy():
    mols = [molecule_from_fixture(load("synthetic_E257.npz"))]
    syn = _run(mols)["syn"]
    e_fe = syn.energy_terms()
    syn.initialize()
    syn.evaluate(force=False, energy=True)
    check_energies(syn.energy_terms()[0], e_fe[0], oracle_magnitudes(mols[0]))
    assert not syn.forces().any()


def test_synthetic_batch_against_oracle():
    """A batch of fresh synthetic molecules (sizes 16-256) against the FP64 oracle."""
    from stormm_b200 import synthetic
    mols = [synthetic.make_molecule(500 + k, n) for k, n in enumerate(
        [16, 23, 31, 32, 33, 47, 64, 65, 96, 127, 128, 129, 200, 255, 256])]
    r = _run(mols)
    f_all = r["forces"]
    off = 0
    for k, m in enumerate(mols):
        o = oracle.from_molecule(m).evaluate(m.coords)
        check_energies(r["energies"][k], o["energies"], oracle_magnitudes(m), m.natom)
        err = rms_rel(f_all[off:off + m.natom], o["forces"])
        assert err <= FORCE_TOL, (m.natom, err)
        off += m.natom


def test_unsupported_model_is_rejected():
    mol = molecule_from_fixture(load("synthetic_E12.npz"))
    with pytest.raises(sb.StormmB200Error):
        sb.Synthesis([mol], igb=7)


def test_clash_mitigated_evaluation_matches_stormm():
    """sb_evaluate_clash (softened Coulomb and Lennard-Jones cores, 1-4 pairs included) against
    STORMM's MM driver with the same clash distance and sigma ratio, on a molecule with close
    contacts; the plain evaluation of the same molecule still matches its plain record."""
    g = load("synthetic_K64.npz")
    mol = molecule_from_fixture(g)
    syn = sb.Synthesis([mol])
    syn.set_coordinates(mol.coords)
    syn.initialize()
    syn.evaluate_clash(float(g["clash_r0"][0]), float(g["clash_ratio"][0]))
    assert syn.status() == 0
    rss = fixture_magnitudes(g)
    check_energies(syn.energy_terms()[0], g["clash_energy_terms"], rss)
    assert rms_rel(syn.forces(), g["clash_frc_total"].reshape(-1, 3)) <= FORCE_TOL
    syn.initialize()
    syn.evaluate()
    check_energies(syn.energy_terms()[0], g["energy_terms_mm"], rss)
    # zero distance and ratio is the plain evaluation, bit for bit
    f_plain = syn.forces_fixed()[0].copy()
    syn.initialize()
    syn.evaluate_clash(0.0, 0.0)
    assert np.array_equal(syn.forces_fixed()[0], f_plain)


def test_neck_gb_on_the_tiled_path_and_without_tables():
    """Neck GB II through the tile-by-tile kernels matches STORMM as the fused kernel does; a
    neck model without its tables is refused."""
    g = load("synthetic_N8.npz")
    mol = molecule_from_fixture(g)
    tiled = _run([mol], tiled_above_atoms=32, **solvent_options(g))
    check_energies(tiled["energies"][0], g["energy_terms"], fixture_magnitudes(g))
    assert rms_rel(tiled["forces"], reference_forces(g)) <= FORCE_TOL
    with pytest.raises(sb.StormmB200Error):
        sb.Synthesis([mol], igb=8)
