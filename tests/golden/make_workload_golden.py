"""Generate tests/golden/workload_single_point_sample.npz by running STORMM's own CPU build on a
sample of the batched single-point workload (1,024 synthetic molecules of 16-256 atoms, OBC-II).

Requires the reference CPU build (oracle/ref/Makefile: oracle/_ref/stormm_ref_driver).  Run
from the repository root:

    python tests/golden/make_workload_golden.py

The sample is every 16th molecule of the workload (64 molecules, indices 0, 16, ..., 1008).
Each is written as Amber prmtop / inpcrd, read back by STORMM's AtomGraph, its coordinates
rounded to the 2^-32 A fixed-point grid, and evaluated by STORMM's FP64 CPU evaluators.  The
fixture keeps, per molecule: its workload index and atom count, the coordinates STORMM used, its
per-term FP64 energies (bond, angle, proper and improper dihedral, LJ, LJ 1-4, Coulomb, Coulomb
1-4, GB) and the total forces of STORMM's MM driver (evalRestrainedMMGB).  The generator checks
that STORMM's parse of each topology equals the molecule the library builds from the same seed
(charges, Lennard-Jones tables, GB radii and screening factors, valence parameters), so a test
can rebuild the molecules from the seed and the sample's coordinates.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import DRIVER, eval_molecule  # noqa: E402
from stormm_b200 import synthetic  # noqa: E402

OUT = os.path.join(HERE, "workload_single_point_sample.npz")
STRIDE = 16


def _same_topology(rec, mol):
    """STORMM's parse of the written topology against the generator's molecule."""
    n = mol.natom
    nt = mol.n_lj_types
    # STORMM's own text-to-number conversion differs from strtod by one ulp on some radii and
    # bond parameters, and the prmtop lists bonds to hydrogen apart from the others, so bonds
    # compare as sets
    ours = sorted(zip(np.minimum(mol.bonds[:, 0], mol.bonds[:, 1]),
                      np.maximum(mol.bonds[:, 0], mol.bonds[:, 1]), mol.bond_k, mol.bond_r0))
    theirs = sorted(zip(np.minimum(rec["bond_i"], rec["bond_j"]),
                        np.maximum(rec["bond_i"], rec["bond_j"]), rec["bond_k"], rec["bond_r0"]))
    checks = {
        "charge": np.array_equal(rec["charge"], mol.charge),
        "pb_radii": np.allclose(rec["pb_radii"], mol.pb_radii, rtol=4e-16, atol=0),
        "gb_screen": np.allclose(rec["gb_screen"], mol.gb_screen, rtol=4e-16, atol=0),
        "lja": np.allclose(rec["lja"].reshape(nt, nt), mol.lja, rtol=1e-15, atol=0),
        "ljb": np.allclose(rec["ljb"].reshape(nt, nt), mol.ljb, rtol=1e-15, atol=0),
        "bonds": len(ours) == len(theirs) and all(
            a[0] == b[0] and a[1] == b[1] and abs(a[2] - b[2]) <= 4e-16 * b[2] and
            abs(a[3] - b[3]) <= 4e-16 * b[3] for a, b in zip(ours, theirs)),
        "natom": int(rec["natom"][0]) == n,
    }
    bad = [k for k, ok in checks.items() if not ok]
    if bad:
        raise RuntimeError(f"STORMM's parse differs from the generator's molecule: {bad}")


def main():
    if not os.path.exists(DRIVER):
        raise SystemExit("build the reference driver first: make -C oracle/ref -j8")
    mols = synthetic.workload_batched_single_point(1024, seed=synthetic.SEED_BASE + 1)
    index = np.arange(0, len(mols), STRIDE)
    natom, coords, forces, terms = [], [], [], []
    with tempfile.TemporaryDirectory() as tmp:
        for k in index:
            mol = mols[k]
            rec, _, _ = eval_molecule(mol, tmp)
            _same_topology(rec, mol)
            natom.append(mol.natom)
            coords.append(rec["coords"].reshape(-1, 3))
            forces.append(rec["frc_total"].reshape(-1, 3))
            terms.append(rec["energy_terms"])
    np.savez_compressed(OUT, index=index.astype(np.int32), natom=np.array(natom, np.int32),
                        coords=np.concatenate(coords), forces=np.concatenate(forces),
                        energy_terms=np.array(terms))
    print("wrote", OUT, len(index), "molecules,", int(np.sum(natom)), "atoms")


if __name__ == "__main__":
    main()
