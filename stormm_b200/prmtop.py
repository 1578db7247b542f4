"""Amber prmtop / inpcrd writer for synthetic molecules.

Writes the sections STORMM's prmtop reader requires (Topology/atomgraph_detailers.cpp:677-1120:
POINTERS, ATOM_NAME, CHARGE, MASS, ATOM_TYPE_INDEX, NUMBER_EXCLUDED_ATOMS, NONBONDED_PARM_INDEX,
RESIDUE_LABEL, RESIDUE_POINTER, BOND / ANGLE / DIHEDRAL parameter and index sections,
SCEE / SCNB scale factors, LENNARD_JONES_ACOEF / BCOEF, EXCLUDED_ATOMS_LIST, HBOND sections,
AMBER_ATOM_TYPE, RADIUS_SET, RADII, SCREEN) in the standard Amber layout.  Charges are written in
Amber's internal units (e * 18.2223).
"""
from __future__ import annotations

import math

import numpy as np

from .synthetic import Molecule

AMBER_CHARGE_SCALE = 18.2223


def _fmt_block(values, per_line, fmt):
    lines = []
    for k in range(0, len(values), per_line):
        lines.append("".join(fmt(v) for v in values[k:k + per_line]))
    if not lines:
        lines.append("")
    return "\n".join(lines) + "\n"


def _section(name, fortran_fmt, values, per_line, fmt):
    return f"%FLAG {name:<74s}\n%FORMAT({fortran_fmt})\n" + _fmt_block(values, per_line, fmt)


def _ints(name, values):
    return _section(name, "10I8", [int(v) for v in values], 10, lambda v: f"{v:8d}")


def _reals(name, values):
    return _section(name, "5E16.8", [float(v) for v in values], 5, lambda v: f"{v:16.8E}")


def _strs(name, values):
    return _section(name, "20a4", list(values), 20, lambda v: f"{v:<4s}"[:4])


def write_prmtop(mol: Molecule, path: str) -> None:
    n = mol.natom
    ntype = mol.n_lj_types
    is_h = mol.z_numbers == 1

    # unique parameter tables (one parameter set per term keeps the mapping trivial)
    nbond = mol.bonds.shape[0]
    nangl = mol.angles.shape[0]
    ndihe = mol.dihedrals.shape[0]

    bonds_h, bonds_x = [], []
    for t in range(nbond):
        i, j = (int(x) for x in mol.bonds[t])
        rec = (3 * i, 3 * j, t + 1)
        (bonds_h if (is_h[i] or is_h[j]) else bonds_x).append(rec)
    angl_h, angl_x = [], []
    for t in range(nangl):
        i, j, k = (int(x) for x in mol.angles[t])
        rec = (3 * i, 3 * j, 3 * k, t + 1)
        (angl_h if (is_h[i] or is_h[j] or is_h[k]) else angl_x).append(rec)
    dihe_h, dihe_x = [], []
    for t in range(ndihe):
        i, j, k, l = (int(x) for x in mol.dihedrals[t])
        # Amber flags "no 1-4" with a negative third index and cannot sign atom 0, so reverse
        # the quartet when k or l is atom 0.
        if k == 0 or l == 0:
            i, j, k, l = l, k, j, i
        kk = -3 * k if not mol.dihe_has14[t] else 3 * k
        rec = (3 * i, 3 * j, kk, 3 * l, t + 1)
        (dihe_h if (is_h[i] or is_h[j] or is_h[k] or is_h[l]) else dihe_x).append(rec)

    # exclusions: each atom lists higher-indexed 1-2, 1-3 and 1-4 partners (1-based), or a 0
    excl_counts, excl_list = [], []
    for i in range(n):
        partners = sorted(j for j in (mol.excl12[i] | mol.excl13[i] | mol.excl14[i]) if j > i)
        if partners:
            excl_counts.append(len(partners))
            excl_list.extend(j + 1 for j in partners)
        else:
            excl_counts.append(1)
            excl_list.append(0)

    # Lennard-Jones tables: NONBONDED_PARM_INDEX points into the packed upper triangle
    nb_index = np.zeros((ntype, ntype), dtype=np.int64)
    acoef, bcoef = [], []
    packed = 0
    for b in range(ntype):
        for a in range(b + 1):
            packed += 1
            nb_index[a, b] = packed
            nb_index[b, a] = packed
            acoef.append(mol.lja[a, b])
            bcoef.append(mol.ljb[a, b])
    # Amber packs (i, j) with i <= j at index j*(j+1)/2 + i (1-based); the loop above yields the
    # same order.
    nb_parm = [int(nb_index[a, b]) for a in range(ntype) for b in range(ntype)]

    names = []
    counters = {}
    for i in range(n):
        el = {1: "H", 6: "C", 7: "N", 8: "O"}.get(int(mol.z_numbers[i]), "X")
        counters[el] = counters.get(el, 0) + 1
        names.append(f"{el}{counters[el] % 1000}")
    atypes = [f"T{int(t)}" for t in mol.lj_idx]

    pointers = [
        n, ntype, len(bonds_h), len(bonds_x), len(angl_h), len(angl_x), len(dihe_h), len(dihe_x),
        0, 0, len(excl_list), 1, len(bonds_x), len(angl_x), len(dihe_x), nbond, nangl, ndihe,
        ntype, 0, 0, 0, 0, 0, 0, 0, 0, 0, n, 0, 0, 0,
    ]
    out = ["%VERSION  VERSION_STAMP = V0001.000  DATE = 12/03/26  00:00:00\n",
           "%FLAG TITLE" + " " * 69 + "\n%FORMAT(20a4)\n" + f"{mol.name:<80s}\n"]
    out.append(_ints("POINTERS", pointers))
    out.append(_strs("ATOM_NAME", names))
    out.append(_reals("CHARGE", mol.charge * AMBER_CHARGE_SCALE))
    out.append(_ints("ATOMIC_NUMBER", mol.z_numbers))
    out.append(_reals("MASS", mol.mass))
    out.append(_ints("ATOM_TYPE_INDEX", mol.lj_idx + 1))
    out.append(_ints("NUMBER_EXCLUDED_ATOMS", excl_counts))
    out.append(_ints("NONBONDED_PARM_INDEX", nb_parm))
    out.append(_strs("RESIDUE_LABEL", ["MOL"]))
    out.append(_ints("RESIDUE_POINTER", [1]))
    out.append(_reals("BOND_FORCE_CONSTANT", mol.bond_k))
    out.append(_reals("BOND_EQUIL_VALUE", mol.bond_r0))
    out.append(_reals("ANGLE_FORCE_CONSTANT", mol.angl_k))
    out.append(_reals("ANGLE_EQUIL_VALUE", mol.angl_theta0))
    out.append(_reals("DIHEDRAL_FORCE_CONSTANT", mol.dihe_amp))
    out.append(_reals("DIHEDRAL_PERIODICITY", mol.dihe_freq))
    out.append(_reals("DIHEDRAL_PHASE", mol.dihe_phase))
    out.append(_reals("SCEE_SCALE_FACTOR", np.full(ndihe, mol.scee)))
    out.append(_reals("SCNB_SCALE_FACTOR", np.full(ndihe, mol.scnb)))
    out.append(_reals("SOLTY", np.zeros(ntype)))
    out.append(_reals("LENNARD_JONES_ACOEF", acoef))
    out.append(_reals("LENNARD_JONES_BCOEF", bcoef))
    out.append(_ints("BONDS_INC_HYDROGEN", [v for r in bonds_h for v in r]))
    out.append(_ints("BONDS_WITHOUT_HYDROGEN", [v for r in bonds_x for v in r]))
    out.append(_ints("ANGLES_INC_HYDROGEN", [v for r in angl_h for v in r]))
    out.append(_ints("ANGLES_WITHOUT_HYDROGEN", [v for r in angl_x for v in r]))
    out.append(_ints("DIHEDRALS_INC_HYDROGEN", [v for r in dihe_h for v in r]))
    out.append(_ints("DIHEDRALS_WITHOUT_HYDROGEN", [v for r in dihe_x for v in r]))
    out.append(_ints("EXCLUDED_ATOMS_LIST", excl_list))
    out.append(_reals("HBOND_ACOEF", []))
    out.append(_reals("HBOND_BCOEF", []))
    out.append(_reals("HBCUT", []))
    out.append(_strs("AMBER_ATOM_TYPE", atypes))
    out.append(_strs("TREE_CHAIN_CLASSIFICATION", ["M"] * n))
    out.append(_ints("JOIN_ARRAY", [0] * n))
    out.append(_ints("IROTAT", [0] * n))
    out.append("%FLAG RADIUS_SET" + " " * 64 + "\n%FORMAT(1a80)\nsynthetic radii (OBC-II)\n")
    out.append(_reals("RADII", mol.pb_radii))
    out.append(_reals("SCREEN", mol.gb_screen))
    out.append(_ints("IPOL", [0]))
    with open(path, "w") as f:
        f.write("".join(out))


def write_inpcrd(mol: Molecule, path: str) -> None:
    c = mol.coords.reshape(-1)
    lines = [f"{mol.name}\n", f"{mol.natom:6d}\n"]
    for k in range(0, c.size, 6):
        lines.append("".join(f"{v:12.7f}" for v in c[k:k + 6]) + "\n")
    with open(path, "w") as f:
        f.write("".join(lines))
