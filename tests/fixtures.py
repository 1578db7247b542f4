"""Helpers that turn golden fixtures into molecule objects for the library and the oracle, and
the energy and force tolerances every GPU test applies.

Tolerances of the FP32 path (FP32 arithmetic, fixed-point accumulation) against FP64 results
(STORMM's CPU build or the FP64 oracle):

* every energy term of every molecule: |E_gpu - E_ref| <= 1e-6 x max(|E_ref|, 1 kcal/mol, R),
  R the root-sum-square of the term's contributions (oracle ``magnitudes``: each bond, angle,
  dihedral, pair or GB self term; a Lennard-Jones pair counts |A|/r^12 + |B|/r^6).  For a term
  whose contributions share a sign R <= |E| and the bound is plain 1e-6 relative (with an
  absolute floor below 1 kcal/mol).  R matters for the Coulomb and Lennard-Jones pair sums and
  GB, differences of large positive and negative parts: on the 1,024-molecule workload one
  241-atom molecule's Coulomb total is -1.6 kcal/mol out of pair terms with R = 620 kcal/mol.
  Each pair evaluated in FP32 is rounded independently (relative 1e-7 or so; r^-12 multiplies
  the rounding of r^2 by six), so the error of the sum grows like R, and 1e-6 of R is what an
  FP32 evaluation of each pair can meet.  The FP64 mode meets the bound without R on every term
  (tests/test_gpu_workloads.py);
* the total energy: within the sum of the per-term bounds;
* forces: RMS relative error at most 5e-6 against FP64.
"""
import glob
import os
from types import SimpleNamespace

import numpy as np

ENERGY_REL_TOL = 1.0e-6
ENERGY_FLOOR = 1.0               # kcal/mol: terms smaller than this are held to 1e-6 kcal/mol
FORCE_TOL = 5.0e-6

from conftest import GOLDEN


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def synthetic_paths():
    return sorted(glob.glob(os.path.join(GOLDEN, "synthetic_*.npz")))


def default_solvent_paths():
    """Synthetic fixtures evaluated with the library's default solvent model (OBC-II,
    dielectric 80, no salt), which can share one synthesis."""
    out = []
    for p in synthetic_paths():
        g = load(os.path.basename(p))
        if (int(g["igb"][0]) == 3 and float(g["dielectric"][0]) == 80.0 and
                float(g["saltcon"][0]) == 0.0):
            out.append(p)
    return out


def reference_paths():
    return sorted(glob.glob(os.path.join(GOLDEN, "reference_*.npz")))


def molecule_from_fixture(g):
    """Topology exactly as STORMM parsed it (charges after smoothing, LJ tables, GB parameters,
    valence terms with their 1-4 attenuation), as the attributes the library expects."""
    n = int(g["natom"][0])
    nt = int(g["n_lj_types"][0])

    def sets(key):
        b, x = g[key + "_bounds"], g[key + "x"]
        return [set(int(v) for v in x[b[i]:b[i + 1]]) for i in range(n)]

    e11 = sets("nb11")
    e12 = sets("nb12")
    e13 = sets("nb13")
    e14 = sets("nb14")
    for i in range(n):
        e12[i] |= e11[i]
    scee = np.asarray(g["dihe_scee"], dtype=np.float64)
    charmm = {}
    if "ubrd_atoms" in g:
        # CHARMM terms (empty for Amber force fields)
        charmm = dict(ubrd_atoms=g["ubrd_atoms"].reshape(-1, 2), ubrd_keq=g["ubrd_keq"],
                      ubrd_leq=g["ubrd_leq"], cimp_atoms=g["cimp_atoms"].reshape(-1, 4),
                      cimp_keq=g["cimp_keq"], cimp_phase=g["cimp_phase"],
                      cmap_atoms=g["cmap_atoms"].reshape(-1, 5), cmap_surface=g["cmap_surface"],
                      cmap_dims=g["cmap_dims"], cmap_values=g["cmap_values"])
    return SimpleNamespace(**charmm,
        natom=n, coords=g["coords"].reshape(n, 3), charge=g["charge"], lj_idx=g["lj_idx"],
        n_lj_types=nt, lja=g["lja"].reshape(nt, nt), ljb=g["ljb"].reshape(nt, nt),
        lja14=g["lja14"].reshape(nt, nt), ljb14=g["ljb14"].reshape(nt, nt),
        excl12=e12, excl13=e13, excl14=e14, pb_radii=g["pb_radii"], gb_screen=g["gb_screen"],
        gb_alpha=g["gb_alpha"], gb_beta=g["gb_beta"], gb_gamma=g["gb_gamma"],
        bonds=np.stack([g["bond_i"], g["bond_j"]], axis=1), bond_k=g["bond_k"],
        bond_r0=g["bond_r0"],
        angles=np.stack([g["angl_i"], g["angl_j"], g["angl_k"]], axis=1), angl_k=g["angl_k_eq"],
        angl_theta0=g["angl_theta0"],
        dihedrals=np.stack([g["dihe_i"], g["dihe_j"], g["dihe_k"], g["dihe_l"]], axis=1),
        dihe_amp=g["dihe_amp"], dihe_freq=g["dihe_freq"], dihe_phase=g["dihe_phase"],
        dihe_has14=scee > 0.0, dihe_scee_array=scee, dihe_scnb_array=g["dihe_scnb"],
        dihe_improper=(np.asarray(g["dihe_kind"]) >= 2).astype(np.int32), scee=1.2, scnb=2.0,
        name="fixture")


def igb_of_fixture(g):
    """Amber igb number of the fixture's implicit solvent model (STORMM enum order)."""
    return {0: 0, 1: 1, 2: 2, 3: 5, 4: 7, 5: 8}[int(g["igb"][0])]


def solvent_options(g):
    """Synthesis options of the fixture's solvent model: igb, dielectric, salt and, for the neck
    models, the neck tables STORMM used."""
    opts = dict(igb=igb_of_fixture(g), dielectric=float(g["dielectric"][0]),
                saltcon=float(g["saltcon"][0]))
    if opts["igb"] in (7, 8):
        opts.update(neck_max_separation=g["neck_max_sep"], neck_max_value=g["neck_max_val"],
                    neck_table_size=int(g["neck_table_size"][0]),
                    neck_cut=float(g["neck_cut"][0]))
    return opts


def reference_forces(g):
    return (g["frc_bond"] + g["frc_angle"] + g["frc_dihedral"] + g["frc_14"] +
            g["frc_nonbonded"] + g["frc_gb"]).reshape(-1, 3)


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def energy_tolerances(e_ref, rss=None, rel=ENERGY_REL_TOL):
    """Per-term bounds (see the module docstring); rss: the oracle's per-term root-sum-squares
    of the contributions, or None for the plain bound rel x max(|E|, 1 kcal/mol)."""
    e_ref = np.asarray(e_ref, dtype=np.float64)
    scale = np.maximum(np.abs(e_ref), ENERGY_FLOOR)
    if rss is not None:
        scale = np.maximum(scale, np.asarray(rss, dtype=np.float64))
    return rel * scale


def energy_excess(e_gpu, e_ref, rss=None, **kw):
    """Error over bound per term (a value above 1 fails)."""
    return np.abs(np.asarray(e_gpu) - np.asarray(e_ref)) / energy_tolerances(e_ref, rss, **kw)


def check_energies(e_gpu, e_ref, rss=None, what="", **kw):
    """Assert every term and the total against the per-term bounds."""
    tol = energy_tolerances(e_ref, rss, **kw)
    err = np.abs(np.asarray(e_gpu) - np.asarray(e_ref))
    assert np.all(err <= tol), (what, err / tol, e_gpu, e_ref)
    assert abs(float(np.sum(e_gpu)) - float(np.sum(e_ref))) <= tol.sum(), what


def total_tolerance(e_ref_terms, rss=None, **kw):
    """Bound on a total energy: the sum of its terms' bounds."""
    return float(energy_tolerances(e_ref_terms, rss, **kw).sum())


def oracle_magnitudes(mol, coords=None):
    """Per-term root-sum-squares of a molecule object at its (or the given) coordinates."""
    import oracle
    return oracle.from_molecule(mol).magnitudes(mol.coords if coords is None else coords)


def fixture_magnitudes(g):
    """Per-term root-sum-squares of a fixture at its coordinates, with STORMM's GB radii."""
    import oracle
    radii = g["gb_radii"] if "gb_radii" in g else None
    return oracle.from_fixture(g).magnitudes(g["coords"], radii)
