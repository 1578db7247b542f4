"""Seeded synthetic molecules for the batched implicit-solvent workloads.

Each molecule is a random tree of heavy atoms with hydrogens filling free valences, built in 3-D
with clash rejection, then parameterised:

* harmonic bonds, k 300-600 kcal/mol/A^2, r0 = the built bond length (1.0-1.54 A);
* harmonic angles, theta0 = 109.5 deg, k 50-80 kcal/mol/rad^2;
* periodic dihedrals, n = 1-3, V 0.1-2 kcal/mol, phase 0 or 180 deg, one term per quartet plus
  an occasional second term that does not carry the 1-4 pair;
* partial charges N(0, 0.3) e shifted to a net charge of exactly zero;
* 8 Lennard-Jones types, sigma 2.0-3.8 A, epsilon 0.02-0.2 kcal/mol, Lorentz-Berthelot mixing;
* 1-2 / 1-3 exclusions, 1-4 pairs scaled 1/1.2 (electrostatic) and 1/2 (Lennard-Jones);
* OBC-II GB radii 1.2-1.9 A and screening factors 0.72-0.85;
* coordinates = built geometry + Gaussian noise.

Polymer-like chains (2,000-5,000 atoms) are a seeded random walk of 1.5 A bond vectors with
nonbonded clash rejection at 2.5 A.

The geometry builder is C++ (csrc/synthetic.cpp, built into libstormm_b200_synth.so); this module
wraps it and defines the seeded workloads.  Parameters are rounded so that an Amber prmtop written
from a molecule (prmtop.py) is read back by STORMM's AtomGraph to exactly the same numbers.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

COULOMB_CONSTANT = 332.0522172900000        # Constants/symbol_values.h:33 (amber_ancient_bioq)
CHARGE_QUANTUM = 2.0 ** -23                 # Topology/atomgraph_constants.h:18


@dataclass
class Molecule:
    """One molecule's topology and coordinates (all indices 0-based, FP64 parameters)."""
    natom: int
    coords: np.ndarray            # (natom, 3) Angstrom
    charge: np.ndarray            # (natom,) e
    lj_idx: np.ndarray            # (natom,) int32, molecule-local type index
    lja: np.ndarray               # (ntype, ntype) A coefficients
    ljb: np.ndarray               # (ntype, ntype) B coefficients
    z_numbers: np.ndarray         # (natom,) int32
    mass: np.ndarray              # (natom,)
    pb_radii: np.ndarray          # (natom,) intrinsic GB radii
    gb_screen: np.ndarray         # (natom,)
    bonds: np.ndarray             # (nbond, 2) int32
    bond_k: np.ndarray
    bond_r0: np.ndarray
    angles: np.ndarray            # (nangl, 3) int32
    angl_k: np.ndarray
    angl_theta0: np.ndarray
    dihedrals: np.ndarray         # (ndihe, 4) int32
    dihe_amp: np.ndarray
    dihe_freq: np.ndarray
    dihe_phase: np.ndarray
    dihe_has14: np.ndarray        # (ndihe,) bool: this term carries the I-L 1-4 pair
    scee: float = 1.2
    scnb: float = 2.0
    name: str = "MOL"
    # derived
    excl12: list = field(default_factory=list)
    excl13: list = field(default_factory=list)
    excl14: list = field(default_factory=list)

    @property
    def n_lj_types(self) -> int:
        return int(self.lja.shape[0])


def _neighbors(natom, bonds):
    nbr = [[] for _ in range(natom)]
    for i, j in bonds:
        nbr[i].append(int(j))
        nbr[j].append(int(i))
    return nbr


def exclusion_lists(natom, bonds):
    """1-2, 1-3 and 1-4 partner sets per atom from the bond graph (STORMM derives the same sets
    from connectivity: Topology/topology_util.cpp, used by static_exclusionmask.cpp:76-100)."""
    nbr = _neighbors(natom, bonds)
    e12 = [set(n) for n in nbr]
    e13 = [set() for _ in range(natom)]
    e14 = [set() for _ in range(natom)]
    for i in range(natom):
        for j in nbr[i]:
            for k in nbr[j]:
                if k != i and k not in e12[i]:
                    e13[i].add(k)
    for i in range(natom):
        for j in nbr[i]:
            for k in nbr[j]:
                if k == i:
                    continue
                for l in nbr[k]:
                    if l != j and l != i and l not in e12[i] and l not in e13[i]:
                        e14[i].add(l)
    return e12, e13, e14



class _SynMolecule(ctypes.Structure):
    _fields_ = [("natom", ctypes.c_int), ("nbond", ctypes.c_int), ("nangl", ctypes.c_int),
                ("ndihe", ctypes.c_int), ("ntype", ctypes.c_int)] + [
        (n, ctypes.POINTER(t)) for n, t in [
            ("coords", ctypes.c_double), ("charge", ctypes.c_double), ("lj_idx", ctypes.c_int),
            ("lja", ctypes.c_double), ("ljb", ctypes.c_double), ("z_numbers", ctypes.c_int),
            ("mass", ctypes.c_double), ("pb_radii", ctypes.c_double),
            ("gb_screen", ctypes.c_double), ("bonds", ctypes.c_int), ("bond_k", ctypes.c_double),
            ("bond_r0", ctypes.c_double), ("angles", ctypes.c_int), ("angl_k", ctypes.c_double),
            ("angl_theta0", ctypes.c_double), ("dihedrals", ctypes.c_int),
            ("dihe_amp", ctypes.c_double), ("dihe_freq", ctypes.c_double),
            ("dihe_phase", ctypes.c_double), ("dihe_has14", ctypes.c_int)]]


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libstormm_b200_synth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"synthetic-molecule library missing: {path} (run the build)")
        _LIB = ctypes.CDLL(path)
        _LIB.sbsyn_make_molecule.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_int, ctypes.POINTER(_SynMolecule)]
        _LIB.sbsyn_make_molecule.restype = ctypes.c_int
        _LIB.sbsyn_free.argtypes = [ctypes.POINTER(_SynMolecule)]
    return _LIB


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _build(seed: int, natom: int, noise: float, kind: int, name: str) -> Molecule:
    lib = _lib()
    m = _SynMolecule()
    rc = lib.sbsyn_make_molecule(ctypes.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), natom, noise, kind,
                                 ctypes.byref(m))
    if rc != 0:
        lib.sbsyn_free(ctypes.byref(m))
        raise RuntimeError(f"synthetic molecule build failed (code {rc}) for natom={natom}")
    try:
        n, nb, na, nd, nt = m.natom, m.nbond, m.nangl, m.ndihe, m.ntype
        bonds = _arr(m.bonds, 2 * nb, np.int32).reshape(-1, 2)
        e12, e13, e14 = exclusion_lists(n, bonds)
        mol = Molecule(
            natom=n, coords=_arr(m.coords, 3 * n, np.float64).reshape(n, 3),
            charge=_arr(m.charge, n, np.float64), lj_idx=_arr(m.lj_idx, n, np.int32),
            lja=_arr(m.lja, nt * nt, np.float64).reshape(nt, nt),
            ljb=_arr(m.ljb, nt * nt, np.float64).reshape(nt, nt),
            z_numbers=_arr(m.z_numbers, n, np.int32), mass=_arr(m.mass, n, np.float64),
            pb_radii=_arr(m.pb_radii, n, np.float64), gb_screen=_arr(m.gb_screen, n, np.float64),
            bonds=bonds, bond_k=_arr(m.bond_k, nb, np.float64),
            bond_r0=_arr(m.bond_r0, nb, np.float64),
            angles=_arr(m.angles, 3 * na, np.int32).reshape(-1, 3),
            angl_k=_arr(m.angl_k, na, np.float64), angl_theta0=_arr(m.angl_theta0, na, np.float64),
            dihedrals=_arr(m.dihedrals, 4 * nd, np.int32).reshape(-1, 4),
            dihe_amp=_arr(m.dihe_amp, nd, np.float64), dihe_freq=_arr(m.dihe_freq, nd, np.float64),
            dihe_phase=_arr(m.dihe_phase, nd, np.float64),
            dihe_has14=_arr(m.dihe_has14, nd, np.int32).astype(bool), name=name,
            excl12=e12, excl13=e13, excl14=e14)
    finally:
        lib.sbsyn_free(ctypes.byref(m))
    return mol


def make_molecule(seed: int, natom: int, noise: float = 0.1, name: str = "MOL") -> Molecule:
    """Seeded random-tree molecule with natom atoms (natom >= 2)."""
    return _build(seed, natom, noise, 0, name)


def make_chain(seed: int, natom: int, noise: float = 0.0, name: str = "CHN") -> Molecule:
    """Seeded polymer-like chain with natom atoms."""
    return _build(seed, natom, noise, 1, name)


# ------------------------------------------------------------------------------------------------
# Workloads.  Seeds are 20261203 + the workload number; molecule k of a workload is built from
# seed (workload_seed * 1000003 + k).
# ------------------------------------------------------------------------------------------------
SEED_BASE = 20261203


def _seed(base: int, k: int) -> int:
    return base * 1000003 + k


def workload_single(seed: int = SEED_BASE) -> list:
    """One 64-atom molecule, 0.1 A coordinate noise."""
    return [make_molecule(_seed(seed, 0), 64, noise=0.1, name="M0")]


def batched_sizes(nsys: int = 1024, seed: int = SEED_BASE + 1) -> np.ndarray:
    return np.random.default_rng(seed).integers(16, 257, size=nsys)


def workload_batched_single_point(nsys: int = 1024, seed: int = SEED_BASE + 1) -> list:
    """1,024 distinct molecules with atom counts uniform on 16-256, 0.1 A noise."""
    sizes = batched_sizes(nsys, seed)
    return [make_molecule(_seed(seed, i), int(n), noise=0.1, name=f"S{i}")
            for i, n in enumerate(sizes)]


def workload_minimization(nsys: int = 4096, seed: int = SEED_BASE + 2) -> list:
    """4,096 molecules with 24-96 atoms, starting coordinates perturbed by 0.3 A noise."""
    sizes = np.random.default_rng(seed).integers(24, 97, size=nsys)
    return [make_molecule(_seed(seed, i), int(n), noise=0.3, name=f"N{i}")
            for i, n in enumerate(sizes)]


def served_sizes(nreq: int, seed: int = SEED_BASE + 3, sigma: float = 0.6) -> np.ndarray:
    """Lognormal request sizes, median 48 atoms, clipped to 12-512 (sigma = 0.6)."""
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(48.0 * np.exp(rng.normal(0.0, sigma, size=nreq))), 12, 512).astype(int)


def workload_served(nreq: int, seed: int = SEED_BASE + 3, sigma: float = 0.6) -> list:
    sizes = served_sizes(nreq, seed, sigma)
    return [make_molecule(_seed(seed, i), int(n), noise=0.3, name=f"R{i}")
            for i, n in enumerate(sizes)]


def workload_chains(nsys: int = 256, seed: int = SEED_BASE + 4) -> list:
    """256 polymer-like chains of 2,000-5,000 atoms."""
    sizes = np.random.default_rng(seed).integers(2000, 5001, size=nsys)
    return [make_chain(_seed(seed, i), int(n), name=f"C{i}") for i, n in enumerate(sizes)]
