"""Amber file intake (sb_read_amber_topology / sb_read_amber_coordinates), host only.

Pinned against STORMM's own parse of its test topologies: the golden fixtures hold the arrays
STORMM's AtomGraph built from Trp-cage and alanine dipeptide (charges, Lennard-Jones tables,
valence terms with their 1-4 factors, 1-2 / 1-3 / 1-4 exclusion lists, atomic numbers, radii and
the per-model GB parameters after setImplicitSolventModel), and the coordinates its PhaseSpace
read.  The files themselves are read from the reference tree when it is present.  Round trips
through this package's prmtop / inpcrd writer cover the rest anywhere.
"""
import os

import numpy as np
import pytest

import stormm_b200 as sb
from stormm_b200 import prmtop as amber_writer
from stormm_b200.synthetic import make_chain, make_molecule

from fixtures import igb_of_fixture, load, molecule_from_fixture, reference_paths

REFERENCE_TEST = os.path.join(os.environ.get("STORMM_REFERENCE_ROOT", "/root/reference"), "test")
FILES = {"trpcage": ("trpcage.top", "trpcage.inpcrd"),
         "ala_dipeptide": ("ala_dipeptide.top", "ala_dipeptide.inpcrd")}


def _canon_bonds(bonds, *params):
    rows = []
    for n, (i, j) in enumerate(np.asarray(bonds)):
        a, b = sorted((int(i), int(j)))
        rows.append((a, b) + tuple(float(p[n]) for p in params))
    return sorted(rows)


def _canon_angles(angles, *params):
    rows = []
    for n, (i, j, k) in enumerate(np.asarray(angles)):
        i, k = (int(i), int(k)) if i < k else (int(k), int(i))
        rows.append((i, int(j), k) + tuple(float(p[n]) for p in params))
    return sorted(rows)


def _canon_dihedrals(dihedrals, *params):
    rows = []
    for n, d in enumerate(np.asarray(dihedrals)):
        fwd = tuple(int(v) for v in d)
        rows.append(min(fwd, fwd[::-1]) + tuple(float(p[n]) for p in params))
    return sorted(rows)


def _rows_close(a, b, natoms, rtol=1e-12):
    assert len(a) == len(b)
    for ra, rb in zip(a, b):
        assert ra[:natoms] == rb[:natoms], (ra, rb)
        np.testing.assert_allclose(ra[natoms:], rb[natoms:], rtol=rtol, atol=1e-12)


def _reference_cases():
    out = []
    for p in reference_paths():
        name = os.path.basename(p)
        system = name[len("reference_"):name.rindex("_igb")]
        out.append((system, name))
    return out


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TEST), reason="reference test files absent")
@pytest.mark.parametrize("system,fixture", _reference_cases())
def test_reader_matches_stormm_parse(system, fixture):
    g = load(fixture)
    ref = molecule_from_fixture(g)
    top, crd = FILES[system]
    igb = igb_of_fixture(g)
    m = sb.read_amber(os.path.join(REFERENCE_TEST, "Topology", top),
                      os.path.join(REFERENCE_TEST, "Trajectory", crd), igb=igb)
    n = ref.natom
    assert m.natom == n
    np.testing.assert_allclose(m.coords, ref.coords, rtol=0, atol=1e-12)
    np.testing.assert_allclose(m.charge, ref.charge, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(m.lj_idx, ref.lj_idx)
    np.testing.assert_array_equal(m.z_numbers, g["z_numbers"])
    np.testing.assert_allclose(m.lja, ref.lja, rtol=1e-14)
    np.testing.assert_allclose(m.ljb, ref.ljb, rtol=1e-14)
    lja14 = getattr(m, "lja14", m.lja)
    ljb14 = getattr(m, "ljb14", m.ljb)
    np.testing.assert_allclose(lja14, ref.lja14, rtol=1e-14)
    np.testing.assert_allclose(ljb14, ref.ljb14, rtol=1e-14)
    # GB parameters after the model's assignment (element screening for the neck models)
    np.testing.assert_allclose(m.pb_radii, ref.pb_radii, rtol=1e-15)   # parsers differ by 1 ulp
    for got, want in ((m.gb_screen, ref.gb_screen), (m.gb_alpha, ref.gb_alpha),
                      (m.gb_beta, ref.gb_beta), (m.gb_gamma, ref.gb_gamma)):
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    # valence terms and their parameters, in any order and atom direction
    _rows_close(_canon_bonds(m.bonds, m.bond_k, m.bond_r0),
                _canon_bonds(ref.bonds, ref.bond_k, ref.bond_r0), 2)
    _rows_close(_canon_angles(m.angles, m.angl_k, m.angl_theta0),
                _canon_angles(ref.angles, ref.angl_k, ref.angl_theta0), 3)
    _rows_close(_canon_dihedrals(m.dihedrals, m.dihe_amp, m.dihe_freq, m.dihe_phase,
                                 m.dihe_scee_array, m.dihe_scnb_array, m.dihe_improper),
                _canon_dihedrals(ref.dihedrals, ref.dihe_amp, ref.dihe_freq, ref.dihe_phase,
                                 ref.dihe_scee_array, ref.dihe_scnb_array, ref.dihe_improper),
                4)
    assert int(g["ninfr14"][0]) == 0
    # exclusions by distance in the bond graph
    for level, want in ((0, ref.excl12), (1, ref.excl13), (2, ref.excl14)):
        got = (m.excl12, m.excl13, m.excl14)[level]
        for a in range(n):
            assert set(got[a]) == set(want[a]), (level, a)
    # STORMM's static exclusion-mask tables from the read topology
    masks = sb.static_exclusion_mask(m)
    np.testing.assert_array_equal(masks["mask_data"], g["se_mask_data"])


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TEST), reason="reference test files absent")
@pytest.mark.parametrize("system", sorted(FILES))
@pytest.mark.parametrize("igb", [1, 2, 5])
def test_read_topology_energies_match_stormm(system, igb):
    """The oracle on the read files reproduces the energies STORMM computed from its own parse
    of the same files (the nine terms this path evaluates)."""
    import oracle
    g = load(f"reference_{system}_igb{igb}.npz")
    top, crd = FILES[system]
    m = sb.read_amber(os.path.join(REFERENCE_TEST, "Topology", top),
                      os.path.join(REFERENCE_TEST, "Trajectory", crd), igb=igb)
    o = oracle.from_molecule(m, igb=igb, dielectric=float(g["dielectric"][0]),
                             saltcon=float(g["saltcon"][0]),
                             coulomb_constant=float(g["coulomb_constant"][0]))
    r = o.evaluate(g["coords"].reshape(-1, 3))
    np.testing.assert_allclose(r["energies"], g["energy_terms"], rtol=1e-9, atol=1e-6)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TEST), reason="reference test files absent")
def test_reader_reports_charmm_terms_and_radius_set():
    m = sb.read_amber(os.path.join(REFERENCE_TEST, "Topology", "ala_dipeptide.top"))
    assert m.cmap_count == 1
    assert m.urey_bradley_count == 0
    assert "mbondi" in m.radius_set
    assert not hasattr(m, "gb_alpha")
    assert np.all(m.coords == 0.0)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TEST), reason="reference test files absent")
@pytest.mark.parametrize("top,fixture", [("ala_dipeptide.top", "charmm_ala_dipeptide.npz"),
                                         ("dhfr_cmap.top", "charmm_dhfr.npz")])
def test_reader_reads_charmm_terms_as_stormm(top, fixture):
    """Urey-Bradley, CHARMM improper and CMAP terms read from the file equal STORMM's parse
    (atoms exactly; parameters and CMAP surface values, column-major, to the last bit of the
    decimal conversion)."""
    m = sb.read_amber(os.path.join(REFERENCE_TEST, "Topology", top))
    g = load(fixture)
    empty = np.zeros(0)
    for key in ("ubrd_atoms", "cimp_atoms", "cmap_atoms", "cmap_surface", "cmap_dims"):
        np.testing.assert_array_equal(np.asarray(getattr(m, key, empty)).reshape(-1),
                                      g[key].reshape(-1), err_msg=key)
    for key in ("ubrd_keq", "ubrd_leq", "cimp_keq", "cimp_phase", "cmap_values"):
        np.testing.assert_allclose(np.asarray(getattr(m, key, empty)), g[key], rtol=1e-15,
                                   atol=0.0, err_msg=key)


@pytest.mark.parametrize("natom,chain", [(2, False), (24, False), (64, True), (200, False)])
def test_round_trip_through_writer(tmp_path, natom, chain):
    src = (make_chain if chain else make_molecule)(seed=1000 + natom, natom=natom)
    top, crd = tmp_path / "m.prmtop", tmp_path / "m.inpcrd"
    amber_writer.write_prmtop(src, str(top))
    amber_writer.write_inpcrd(src, str(crd))
    m = sb.read_amber(top, crd)
    assert m.natom == src.natom
    np.testing.assert_allclose(m.coords, src.coords, rtol=0, atol=6e-8)
    np.testing.assert_allclose(m.charge, src.charge, rtol=1e-8, atol=1e-12)
    np.testing.assert_array_equal(m.lj_idx, src.lj_idx)
    np.testing.assert_array_equal(m.z_numbers, src.z_numbers)
    np.testing.assert_allclose(m.lja, src.lja, rtol=1e-8)
    np.testing.assert_allclose(m.ljb, src.ljb, rtol=1e-8)
    np.testing.assert_allclose(m.pb_radii, src.pb_radii, rtol=1e-8)
    np.testing.assert_allclose(m.gb_screen, src.gb_screen, rtol=1e-8)
    _rows_close(_canon_bonds(m.bonds, m.bond_k, m.bond_r0),
                _canon_bonds(src.bonds, src.bond_k, src.bond_r0), 2, rtol=1e-8)
    _rows_close(_canon_angles(m.angles, m.angl_k, m.angl_theta0),
                _canon_angles(src.angles, src.angl_k, src.angl_theta0), 3, rtol=1e-8)
    has14 = np.asarray(src.dihe_has14, dtype=bool)
    _rows_close(_canon_dihedrals(m.dihedrals, m.dihe_amp, m.dihe_freq, m.dihe_phase,
                                 m.dihe_has14),
                _canon_dihedrals(src.dihedrals, src.dihe_amp, src.dihe_freq, src.dihe_phase,
                                 has14), 4, rtol=1e-8)
    np.testing.assert_allclose(m.dihe_scee_array, np.where(m.dihe_has14, src.scee, 0.0))
    for got, want in ((m.excl12, src.excl12), (m.excl13, src.excl13), (m.excl14, src.excl14)):
        for a in range(src.natom):
            assert set(got[a]) == set(want[a])


def test_gb_parameter_assignment_by_model(tmp_path):
    src = make_molecule(seed=77, natom=40)
    top = tmp_path / "m.prmtop"
    amber_writer.write_prmtop(src, str(top))
    obc2 = sb.read_amber(top, igb=sb.SB_GB_OBC2)
    assert np.all(obc2.gb_alpha == 1.0) and np.all(obc2.gb_beta == 0.8)
    assert np.all(obc2.gb_gamma == 4.85)
    np.testing.assert_allclose(obc2.gb_screen, src.gb_screen, rtol=1e-8)   # kept from the file
    hct = sb.read_amber(top, igb=sb.SB_GB_HCT)
    assert np.all(hct.gb_alpha == 0.0)
    gbn2 = sb.read_amber(top, igb=sb.SB_GB_NECK2)
    hydrogens = src.z_numbers == 1
    assert np.all(gbn2.gb_screen[hydrogens] == 1.425952)
    assert np.all(gbn2.gb_alpha[hydrogens] == 0.788440)


def test_errors(tmp_path):
    with pytest.raises(sb.StormmB200Error, match="cannot open"):
        sb.read_amber(tmp_path / "missing.prmtop")
    bad = tmp_path / "bad.prmtop"
    bad.write_text("not a topology\n")
    with pytest.raises(sb.StormmB200Error, match="FLAG"):
        sb.read_amber(bad)
    # a unit cell is recorded and not applied: this path is non-periodic
    src = make_molecule(seed=5, natom=12)
    top = tmp_path / "box.prmtop"
    amber_writer.write_prmtop(src, str(top))
    lines = top.read_text().split("\n")
    k = next(i for i, ln in enumerate(lines) if ln.startswith("%FLAG POINTERS")) + 2
    fields = [lines[k + 2][c:c + 8] for c in range(0, 80, 8)]      # pointers 21-30
    fields[7] = "%8d" % 1                                            # IFBOX, pointer 28
    lines[k + 2] = "".join(fields)
    top.write_text("\n".join(lines))
    assert sb.read_amber(top).unit_cell == 1     # recorded, not applied
    crd = tmp_path / "m.inpcrd"
    amber_writer.write_inpcrd(src, str(crd))
    with pytest.raises(sb.StormmB200Error, match="atoms"):
        sb.read_amber_coordinates(crd, src.natom + 1)
    ok = tmp_path / "ok.prmtop"
    amber_writer.write_prmtop(src, str(ok))
    with pytest.raises(sb.StormmB200Error, match="unknown GB model"):
        sb.read_amber(ok, igb=3)


DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                      "_ref", "stormm_ref_driver")
MORE_FILES = ["biotin", "drug_example_dry", "med_1", "med_3", "dna", "rna", "symmetry_C3",
              "stereo_L1", "hydrogenate", "bromobenzene", "dhfr_cmap"]


@pytest.mark.skipif(not (os.path.isdir(REFERENCE_TEST) and os.path.exists(DRIVER)),
                    reason="reference test files or the reference driver absent")
@pytest.mark.parametrize("name", MORE_FILES)
def test_reader_on_more_stormm_topologies(tmp_path, name):
    """More of the reference's own test topologies (small drug-like molecules, nucleic acids,
    a 2,730-atom protein, a CMAP protein), read here and by STORMM's AtomGraph through the
    reference driver at the same time: the oracle on our parse reproduces STORMM's nine energy
    terms on its parse to 1e-9 relative, and the 1-2 / 1-3 / 1-4 exclusions are the same."""
    import subprocess
    import oracle
    sys_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    import sys
    if sys_path not in sys.path:
        sys.path.insert(0, sys_path)
    from make_golden import read_records
    top = os.path.join(REFERENCE_TEST, "Topology", name + ".top")
    crd = os.path.join(REFERENCE_TEST, "Trajectory", name + ".inpcrd")
    out = str(tmp_path / "rec.bin")
    r = subprocess.run([DRIVER, "eval", top, crd, out, "--igb", "5", "--qtol", "1e-10",
                        "--qdisc", "9.31322574615478515625E-10"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = read_records(out)
    m = sb.read_amber(top, crd, igb=5)
    assert m.natom == int(g["natom"][0])
    for key, got in (("nb12", m.excl12), ("nb13", m.excl13), ("nb14", m.excl14)):
        b, x = g[key + "_bounds"], g[key + "x"]
        for a in range(m.natom):
            assert set(got[a]) == set(int(v) for v in x[b[a]:b[a + 1]]), (key, a)
    o = oracle.from_molecule(m, igb=5, dielectric=float(g["dielectric"][0]),
                             saltcon=float(g["saltcon"][0]),
                             coulomb_constant=float(g["coulomb_constant"][0]))
    e = o.evaluate(g["coords"].reshape(-1, 3), forces=False)["energies"]
    ref = g["energy_terms"]
    # STORMM's own GB energy of the DNA file comes out NaN in this driver: compare what it
    # computed as a number
    ok = np.isfinite(ref)
    assert ok[:8].all()
    scale = max(np.abs(ref[ok]).sum(), 10.0)
    assert np.all(np.abs(e[ok] - ref[ok]) <= 1e-9 * scale), (e, ref)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TEST), reason="reference test files absent")
def test_reader_refuses_virtual_sites():
    with pytest.raises(sb.StormmB200Error, match="virtual sites"):
        sb.read_amber(os.path.join(REFERENCE_TEST, "Topology", "ahector.top"))
