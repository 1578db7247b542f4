"""Generate tests/golden/conformer_geometry.npz with STORMM's own CPU build: its clash verdicts
(detectClash, Structure/clash_detection.tpp) and mass-weighted aligned RMSDs (RMSDMethod::
ALIGN_MASS, Structure/rmsd.h) on geometries of synthetic molecules, the two ingredients of the
conformer application's selection (apps/Conf/src/analysis.cpp:75-237).

Requires the reference CPU build (oracle/ref/Makefile: oracle/_ref/stormm_ref_driver).  Run from
the repository root:

    python tests/golden/make_conformer_golden.py

Two molecules, of 48 and 24 atoms (detectClash tests molecules of at least 32 atoms through a
spatial grid, smaller ones directly).  Geometries: the molecule itself, replicas from
stormm_b200.conformers.ConformerSearch (no clash by construction), replicas turned about their
rotatable bonds without the clash check (some clash), and copies with one atom moved onto a
neighbour at 0.15-2.0 A (clashes on either side of the limits).  Each is written as an Amber coordinate file and read back; the fixture keeps the
coordinates as read, STORMM's verdicts and its RMSDs against the first geometry.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import DRIVER, read_records  # noqa: E402
import stormm_b200 as sb  # noqa: E402
from stormm_b200 import conformers, prmtop, synthetic  # noqa: E402

CASES = [(7272, 48), (7273, 24)]    # (seed, atoms): detectClash's grid path, its direct path


def geometries(mol):
    rng = np.random.default_rng(5)
    out = [mol.coords]
    search = conformers.ConformerSearch(mol, replicas=20, seed=9)
    out.extend(search.start)
    bonds = conformers.rotatable_bonds(mol.natom, mol.bonds)
    for _ in range(30):
        xyz = np.array(mol.coords, dtype=np.float64, copy=True)
        for (i, j, moved) in bonds:
            xyz = conformers.rotate_about_bond(xyz, i, j, moved, rng.uniform(0.0, 2.0 * np.pi))
        out.append(xyz)
    for _ in range(20):
        xyz = np.array(mol.coords, dtype=np.float64, copy=True)
        a, b = rng.choice(mol.natom, size=2, replace=False)
        d = xyz[a] - xyz[b]
        xyz[a] = xyz[b] + d / np.linalg.norm(d) * rng.uniform(0.15, 2.0)
        out.append(xyz)
    return out


def main():
    arrays = {}
    for c, (seed, natom) in enumerate(CASES):
        mol = synthetic.make_molecule(synthetic._seed(seed, 0), natom, noise=0.1, name="conf")
        with tempfile.TemporaryDirectory() as tmp:
            top = os.path.join(tmp, "m.top")
            prmtop.write_prmtop(mol, top)
            paths, coords = [], []
            for k, xyz in enumerate(geometries(mol)):
                m = synthetic.Molecule(**{**mol.__dict__, "coords": xyz})
                p = os.path.join(tmp, f"g{k}.crd")
                prmtop.write_inpcrd(m, p)
                paths.append(p)
                coords.append(sb.read_amber_coordinates(p, mol.natom))
            lst = os.path.join(tmp, "list.txt")
            with open(lst, "w") as f:
                f.write("\n".join(paths) + "\n")
            out = os.path.join(tmp, "geo.bin")
            subprocess.run([DRIVER, "geometry", top, lst, out], check=True, capture_output=True)
            rec = read_records(out)
        arrays.update({f"seed{c}": seed, f"natom{c}": natom, f"coords{c}": np.stack(coords),
                       f"clash{c}": rec["clash"], f"rmsd{c}": rec["rmsd_to_first"]})
        print(f"{natom} atoms: {len(coords)} geometries, {int(rec['clash'].sum())} clashing")
    np.savez_compressed(os.path.join(HERE, "conformer_geometry.npz"), cases=len(CASES), **arrays)


if __name__ == "__main__":
    main()
