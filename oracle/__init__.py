"""ctypes binding to the FP64 CPU oracle (stormm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg as the checker of the CUDA path, never by the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
NTERMS = 9
TERM_NAMES = ["bond", "angle", "proper_dihedral", "improper_dihedral", "vdw", "vdw_14",
              "elec", "elec_14", "gb"]


def build(force: bool = False) -> str:
    """Compile stormm_oracle.c into liboracle.so beside it."""
    src = os.path.join(HERE, "stormm_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-o", LIB_PATH, src, "-lm"],
                       check=True)
    return LIB_PATH


class _System(ctypes.Structure):
    _fields_ = [
        ("natom", ctypes.c_int), ("coulomb_constant", ctypes.c_double),
        ("charge", ctypes.c_void_p), ("lj_idx", ctypes.c_void_p), ("n_lj_types", ctypes.c_int),
        ("lja", ctypes.c_void_p), ("ljb", ctypes.c_void_p), ("lja14", ctypes.c_void_p),
        ("ljb14", ctypes.c_void_p), ("excl_bounds", ctypes.c_void_p),
        ("excl_list", ctypes.c_void_p), ("igb", ctypes.c_int), ("dielectric", ctypes.c_double),
        ("saltcon", ctypes.c_double), ("pb_radii", ctypes.c_void_p), ("gb_screen", ctypes.c_void_p),
        ("gb_alpha", ctypes.c_void_p), ("gb_beta", ctypes.c_void_p), ("gb_gamma", ctypes.c_void_p),
        ("nbond", ctypes.c_int), ("bond_i", ctypes.c_void_p), ("bond_j", ctypes.c_void_p),
        ("bond_k", ctypes.c_void_p), ("bond_r0", ctypes.c_void_p),
        ("nangl", ctypes.c_int), ("angl_i", ctypes.c_void_p), ("angl_j", ctypes.c_void_p),
        ("angl_k", ctypes.c_void_p), ("angl_keq", ctypes.c_void_p),
        ("angl_theta0", ctypes.c_void_p),
        ("ndihe", ctypes.c_int), ("dihe_i", ctypes.c_void_p), ("dihe_j", ctypes.c_void_p),
        ("dihe_k", ctypes.c_void_p), ("dihe_l", ctypes.c_void_p), ("dihe_amp", ctypes.c_void_p),
        ("dihe_freq", ctypes.c_void_p), ("dihe_phase", ctypes.c_void_p),
        ("dihe_scee", ctypes.c_void_p), ("dihe_scnb", ctypes.c_void_p),
        ("dihe_improper", ctypes.c_void_p), ("neck_idx", ctypes.c_void_p),
        ("neck_table_size", ctypes.c_int), ("neck_max_sep", ctypes.c_void_p),
        ("neck_max_val", ctypes.c_void_p), ("neck_cut", ctypes.c_double),
    ]


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        build()
        _LIB = ctypes.CDLL(LIB_PATH)
        _LIB.orc_evaluate.argtypes = [ctypes.POINTER(_System)] + [ctypes.c_void_p] * 6 + [
            ctypes.c_int]
        _LIB.orc_minimize.argtypes = [ctypes.POINTER(_System), ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        _LIB.orc_minimize_ex.argtypes = [ctypes.POINTER(_System), ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        _LIB.orc_evaluate_clash.argtypes = [ctypes.POINTER(_System)] + [ctypes.c_void_p] * 6 + [
            ctypes.c_int, ctypes.c_double, ctypes.c_double]
        _LIB.orc_minimize_clash.argtypes = [ctypes.POINTER(_System), ctypes.c_void_p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_int)]
        _LIB.orc_energy_magnitudes.argtypes = [ctypes.POINTER(_System)] + [ctypes.c_void_p] * 3
        _LIB.orc_float_to_int63.argtypes = [ctypes.c_float, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int32)]
        _LIB.orc_double_to_int95.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(ctypes.c_int32)]
    return _LIB


class OracleSystem:
    """Holds contiguous arrays for one molecule and the orc_system struct pointing at them."""

    def __init__(self, **arrays):
        self._keep = {}
        s = _System()
        for name, ctype in _System._fields_:
            if ctype is ctypes.c_void_p:
                if name not in arrays or arrays[name] is None:
                    setattr(s, name, None)
                    continue
                dt = np.int32 if name in ("lj_idx", "excl_bounds", "excl_list", "bond_i",
                                          "bond_j", "angl_i", "angl_j", "angl_k", "dihe_i",
                                          "dihe_j", "dihe_k", "dihe_l",
                                          "dihe_improper", "neck_idx") else np.float64
                a = np.ascontiguousarray(np.asarray(arrays[name]).reshape(-1), dtype=dt)
                self._keep[name] = a
                setattr(s, name, a.ctypes.data)
            else:
                setattr(s, name, arrays.get(name, 0))
        self.struct = s
        self.natom = int(arrays["natom"])

    def evaluate(self, coords, forces=True, terms=7, clash_distance=0.0, clash_ratio=0.0):
        """Energies (and forces); with clash_distance or clash_ratio positive, the
        clash-mitigated evaluation (softened Coulomb and Lennard-Jones cores)."""
        lib = _lib()
        c = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1))
        e = np.zeros(NTERMS)
        f = np.zeros(3 * self.natom) if forces else None
        psi = np.zeros(self.natom)
        rad = np.zeros(self.natom)
        sde = np.zeros(self.natom)
        lib.orc_evaluate_clash(ctypes.byref(self.struct), c.ctypes.data,
                               f.ctypes.data if f is not None else None, e.ctypes.data,
                               psi.ctypes.data, rad.ctypes.data, sde.ctypes.data, terms,
                               clash_distance, clash_ratio)
        return {"energies": e, "forces": None if f is None else f.reshape(-1, 3), "psi": psi,
                "radii": rad, "sumdeijda": sde}

    def magnitudes(self, coords, radii=None):
        """Per-term sum of the absolute values of the contributions (orc_energy_magnitudes);
        radii: the effective GB radii of these coordinates (evaluated here when omitted)."""
        lib = _lib()
        c = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1))
        if radii is None:
            radii = self.evaluate(coords, forces=False)["radii"]
        rad = np.ascontiguousarray(np.asarray(radii, dtype=np.float64))
        m = np.zeros(NTERMS)
        lib.orc_energy_magnitudes(ctypes.byref(self.struct), c.ctypes.data, rad.ctypes.data,
                                  m.ctypes.data)
        return m

    def minimize(self, coords, maxcyc, sd_cycles, dx0=0.01, drms=0.0, with_cycles=False,
                 clash_cycles=0, clash_distance=0.2, clash_ratio=0.5):
        """Line minimization; the first clash_cycles cycles clash-damped (STORMM's defaults
        for the distance and the ratio)."""
        lib = _lib()
        c = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1)).copy()
        hist = np.zeros(maxcyc + 1)
        ran = ctypes.c_int(0)
        lib.orc_minimize_clash(ctypes.byref(self.struct), c.ctypes.data, maxcyc, sd_cycles, dx0,
                               drms, clash_cycles, clash_distance, clash_ratio,
                               hist.ctypes.data, ctypes.byref(ran))
        if with_cycles:
            return c.reshape(-1, 3), hist, ran.value
        return c.reshape(-1, 3), hist


def _csr_from_sets(natom, sets_list):
    bounds = np.zeros(natom + 1, dtype=np.int32)
    items = []
    for i in range(natom):
        s = set()
        for sets in sets_list:
            s |= set(sets[i])
        s.discard(i)
        items.extend(sorted(s))
        bounds[i + 1] = len(items)
    return bounds, np.array(items, dtype=np.int32)


def from_fixture(g) -> OracleSystem:
    """Oracle system from a golden fixture (parameters as STORMM parsed them)."""
    n = int(g["natom"][0])
    sets = []
    for key in ("nb11", "nb12", "nb13", "nb14"):
        b, x = g[key + "_bounds"], g[key + "x"]
        sets.append([x[b[i]:b[i + 1]] for i in range(n)])
    eb, el = _csr_from_sets(n, sets)
    igb_enum = int(g["igb"][0])
    # STORMM's ImplicitSolventModel enumeration: NONE, HCT_GB, OBC_GB, OBC_GB_II, NECK_GB,
    # NECK_GB_II
    igb = {0: 0, 1: 1, 2: 2, 3: 5, 4: 7, 5: 8}[igb_enum]
    neck = {}
    if igb in (7, 8):
        neck = dict(neck_idx=g["neck_gb_idx"], neck_table_size=int(g["neck_table_size"][0]),
                    neck_max_sep=g["neck_max_sep"], neck_max_val=g["neck_max_val"],
                    neck_cut=float(g["neck_cut"][0]))
    return OracleSystem(**neck,
        natom=n, coulomb_constant=float(g["coulomb_constant"][0]), charge=g["charge"],
        lj_idx=g["lj_idx"], n_lj_types=int(g["n_lj_types"][0]), lja=g["lja"], ljb=g["ljb"],
        lja14=g["lja14"], ljb14=g["ljb14"], excl_bounds=eb, excl_list=el, igb=igb,
        dielectric=float(g["dielectric"][0]), saltcon=float(g["saltcon"][0]),
        pb_radii=g["pb_radii"], gb_screen=g["gb_screen"], gb_alpha=g["gb_alpha"],
        gb_beta=g["gb_beta"], gb_gamma=g["gb_gamma"],
        nbond=len(g["bond_i"]), bond_i=g["bond_i"], bond_j=g["bond_j"], bond_k=g["bond_k"],
        bond_r0=g["bond_r0"], nangl=len(g["angl_i"]), angl_i=g["angl_i"], angl_j=g["angl_j"],
        angl_k=g["angl_k"], angl_keq=g["angl_k_eq"], angl_theta0=g["angl_theta0"],
        ndihe=len(g["dihe_i"]), dihe_i=g["dihe_i"], dihe_j=g["dihe_j"], dihe_k=g["dihe_k"],
        dihe_l=g["dihe_l"], dihe_amp=g["dihe_amp"], dihe_freq=g["dihe_freq"],
        dihe_phase=g["dihe_phase"], dihe_scee=g["dihe_scee"], dihe_scnb=g["dihe_scnb"],
        dihe_improper=(np.asarray(g["dihe_kind"]) >= 2).astype(np.int32))


def from_molecule(m, igb: int = 5, dielectric: float = 80.0, saltcon: float = 0.0,
                  coulomb_constant: float = 332.0522172900000) -> OracleSystem:
    """Oracle system from a Molecule: a synthetic one (one scee / scnb, no impropers, OBC-II
    alpha / beta / gamma = 1.0, 0.8, 4.85 by model) or one read from an Amber topology, whose
    per-dihedral 1-4 factors, improper flags, 1-4 Lennard-Jones tables and per-atom GB
    parameters are used when present."""
    if igb in (7, 8):
        raise ValueError("neck GB needs the neck tables: build the oracle system from a fixture")
    n = m.natom
    eb, el = _csr_from_sets(n, [m.excl12, m.excl13, m.excl14])
    ab = {1: (0.0, 0.0, 0.0), 2: (0.8, 0.0, 2.909125), 5: (1.0, 0.8, 4.85)}.get(igb, (0, 0, 0))
    has14 = np.asarray(m.dihe_has14, dtype=bool)
    nd = m.dihedrals.shape[0]
    scee = getattr(m, "dihe_scee_array", None)
    scnb = getattr(m, "dihe_scnb_array", None)
    improper = getattr(m, "dihe_improper", None)
    alpha = getattr(m, "gb_alpha", None)
    beta = getattr(m, "gb_beta", None)
    gamma = getattr(m, "gb_gamma", None)
    return OracleSystem(
        natom=n, coulomb_constant=coulomb_constant, charge=m.charge, lj_idx=m.lj_idx,
        n_lj_types=m.n_lj_types, lja=m.lja, ljb=m.ljb, lja14=getattr(m, "lja14", m.lja),
        ljb14=getattr(m, "ljb14", m.ljb), excl_bounds=eb, excl_list=el, igb=igb,
        dielectric=dielectric, saltcon=saltcon, pb_radii=m.pb_radii, gb_screen=m.gb_screen,
        gb_alpha=alpha if alpha is not None else np.full(n, ab[0]),
        gb_beta=beta if beta is not None else np.full(n, ab[1]),
        gb_gamma=gamma if gamma is not None else np.full(n, ab[2]),
        nbond=m.bonds.shape[0], bond_i=m.bonds[:, 0], bond_j=m.bonds[:, 1], bond_k=m.bond_k,
        bond_r0=m.bond_r0, nangl=m.angles.shape[0], angl_i=m.angles[:, 0],
        angl_j=m.angles[:, 1], angl_k=m.angles[:, 2], angl_keq=m.angl_k,
        angl_theta0=m.angl_theta0, ndihe=nd, dihe_i=m.dihedrals[:, 0],
        dihe_j=m.dihedrals[:, 1], dihe_k=m.dihedrals[:, 2], dihe_l=m.dihedrals[:, 3],
        dihe_amp=m.dihe_amp, dihe_freq=m.dihe_freq, dihe_phase=m.dihe_phase,
        dihe_scee=scee if scee is not None else np.where(has14, m.scee, 0.0),
        dihe_scnb=scnb if scnb is not None else np.where(has14, m.scnb, 0.0),
        dihe_improper=(np.asarray(improper, dtype=np.int32) if improper is not None else
                       np.zeros(nd, dtype=np.int32)))


def float_to_int63(v: float):
    x, y = ctypes.c_int32(), ctypes.c_int32()
    _lib().orc_float_to_int63(v, ctypes.byref(x), ctypes.byref(y))
    return x.value, y.value


def double_to_int95(v: float):
    x, y = ctypes.c_int64(), ctypes.c_int32()
    _lib().orc_double_to_int95(v, ctypes.byref(x), ctypes.byref(y))
    return x.value, y.value


def sasa_radii(m) -> np.ndarray:
    """Per-atom surface-area radii as STORMM's surface area takes them
    (Potential/surface_area.tpp:163-173): half the sigma of the first n_lj_types entries of the
    pair table, i.e. of (type 0, atom type), sigma = sqrt(cbrt(A / B)) with B > 1e-6
    (Topology/atomgraph_detailers.cpp:270-277)."""
    a = np.asarray(m.lja, dtype=np.float64).reshape(-1)[np.asarray(m.lj_idx)]
    b = np.asarray(m.ljb, dtype=np.float64).reshape(-1)[np.asarray(m.lj_idx)]
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(b > 1e-6, 0.5 * np.sqrt(np.cbrt(a / np.where(b > 0, b, 1.0))), 0.0)


def surface_area(coords, radii, points, probe=1.4, weight=1.0) -> float:
    """STORMM's sphere-point surface area (Potential/surface_area.tpp:28-161): cells of at least
    twice the largest enlarged radius over the bounding box, a point of an atom in cell (i, j, k)
    tested against atoms in cells i-1..i, j-1..j, k-1..k only, strict inequality, zero when an
    axis has no extent."""
    x = np.asarray(coords, dtype=np.float64)
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    origin = x.min(axis=0)
    length = x.max(axis=0) - origin
    width_min = 2.0 * (radii.max() + probe)
    count = np.ceil(length / width_min).astype(int)
    if (count == 0).any():
        return 0.0
    width = length / count
    cell = np.clip(((x - origin) / width).astype(int), 0, count - 1)
    r_eff = radii + probe
    patch = 4.0 * np.pi / len(pts)
    total = 0.0
    for m in range(len(x)):
        near = np.all((cell <= cell[m]) & (cell >= cell[m] - 1), axis=1)
        near[m] = False
        p = x[m] + pts * r_eff[m]
        d = p[:, None, :] - x[near][None, :, :]
        d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
        buried = (d2 < r_eff[near][None, :] ** 2).any(axis=1)
        total += np.count_nonzero(~buried) * (patch * r_eff[m] * r_eff[m])
    return total * weight
