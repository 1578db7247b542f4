"""stormm_b200: B200-native batched implicit-solvent molecular mechanics.

Python access to the C ABI of include/stormm_b200.h (libstormm_b200.so, built in-tree by
stormm_b200/build.py).  The library is the product; this module only marshals arguments.  There
is no CPU fallback: if the CUDA library is missing or no device is usable, every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libstormm_b200.so")

SB_OK = 0
SB_GB_NONE, SB_GB_HCT, SB_GB_OBC, SB_GB_OBC2, SB_GB_NECK, SB_GB_NECK2 = 0, 1, 2, 5, 7, 8
TERM_VALENCE, TERM_NONBONDED, TERM_GB, TERM_ALL = 1, 2, 4, 7
TUNE_EVALUATE, TUNE_MINIMIZE = 1, 2
MIN_GRAPH, MIN_PERSISTENT = 0, 1
PRECISION_SINGLE, PRECISION_DOUBLE = 0, 1
# AtomicRadiusSet (STORMM Topology/atomgraph_enumerators.h:150-152)
RADII_NONE, RADII_BONDI, RADII_AMBER6, RADII_MBONDI, RADII_MBONDI2, RADII_MBONDI3, RADII_PARSE = \
    range(7)
INIT_FORCES, INIT_ENERGIES, INIT_GB_WORKSPACE = 1, 2, 4
SB_REQUEST_MINIMIZE, SB_REQUEST_EVALUATE = 0, 1
NRG_STRIDE = 16
# StateVariable slots (STORMM Potential/energy_enumerators.h:36-50)
NRG_SLOTS = {"bond": 0, "angle": 1, "proper_dihedral": 2, "improper_dihedral": 3,
             "urey_bradley": 4, "charmm_improper": 5, "cmap": 6, "vdw": 7, "vdw_14": 8,
             "elec": 9, "elec_14": 10, "gb": 11, "restraint": 12}
# order of the oracle's / reference driver's nine energy terms
TERM_ORDER = ["bond", "angle", "proper_dihedral", "improper_dihedral", "vdw", "vdw_14", "elec",
              "elec_14", "gb"]

_P = ctypes.c_void_p


class Topology(ctypes.Structure):
    _fields_ = [
        ("natom", ctypes.c_int), ("charge", _P), ("lj_idx", _P), ("n_lj_types", ctypes.c_int),
        ("lja", _P), ("ljb", _P), ("lja14", _P), ("ljb14", _P), ("excl_bounds", _P),
        ("excl_list", _P), ("pb_radii", _P), ("gb_screen", _P), ("gb_alpha", _P),
        ("gb_beta", _P), ("gb_gamma", _P), ("nbond", ctypes.c_int), ("bond_atoms", _P),
        ("bond_keq", _P), ("bond_leq", _P), ("nangl", ctypes.c_int), ("angl_atoms", _P),
        ("angl_keq", _P), ("angl_theta0", _P), ("ndihe", ctypes.c_int), ("dihe_atoms", _P),
        ("dihe_amp", _P), ("dihe_freq", _P), ("dihe_phase", _P), ("dihe_scee", _P),
        ("dihe_scnb", _P), ("dihe_improper", _P),
        ("nubrd", ctypes.c_int), ("ubrd_atoms", _P), ("ubrd_keq", _P), ("ubrd_leq", _P),
        ("ncimp", ctypes.c_int), ("cimp_atoms", _P), ("cimp_keq", _P), ("cimp_phase", _P),
        ("ncmap", ctypes.c_int), ("cmap_atoms", _P), ("cmap_surface", _P),
        ("ncmap_surf", ctypes.c_int), ("cmap_dims", _P), ("cmap_values", _P),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("igb", ctypes.c_int), ("dielectric", ctypes.c_double), ("saltcon", ctypes.c_double),
        ("coulomb_constant", ctypes.c_double), ("gpos_bits", ctypes.c_int),
        ("frc_bits", ctypes.c_int), ("nrg_bits", ctypes.c_int),
        ("max_atoms_per_unit", ctypes.c_int), ("max_tiles_per_unit", ctypes.c_int),
        ("threads_per_block", ctypes.c_int), ("device", ctypes.c_int),
        ("tiled_above_atoms", ctypes.c_int), ("precision", ctypes.c_int),
        ("neck_max_separation", ctypes.c_void_p), ("neck_max_value", ctypes.c_void_p),
        ("neck_table_size", ctypes.c_int), ("neck_cut", ctypes.c_double),
    ]


VWU_TASKS = ["BOND", "ANGL", "DIHE", "UBRD", "CBND", "CIMP", "CDHE", "CMAP", "INFR14", "RPOSN",
             "RBOND", "RANGL", "RDIHE", "VSITE", "SETTLE", "CGROUP"]


class ValenceTopology(ctypes.Structure):
    _fields_ = [
        ("natom", ctypes.c_int), ("z_numbers", _P), ("nb12_bounds", _P), ("nb12_list", _P),
        ("solvent", _P),
        ("nbond", ctypes.c_int), ("bond_i", _P), ("bond_j", _P), ("bond_param", _P),
        ("bond_relevance", _P),
        ("nangl", ctypes.c_int), ("angl_i", _P), ("angl_j", _P), ("angl_k", _P),
        ("angl_param", _P), ("angl_relevance", _P),
        ("ndihe", ctypes.c_int), ("dihe_i", _P), ("dihe_j", _P), ("dihe_k", _P), ("dihe_l", _P),
        ("dihe_param", _P), ("dihe14_param", _P), ("dihe_kind", _P),
        ("ninfr14", ctypes.c_int), ("infr14_i", _P), ("infr14_l", _P), ("infr14_param", _P),
        ("nsettle", ctypes.c_int), ("settle_ox", _P), ("settle_h1", _P), ("settle_h2", _P),
        ("settle_param", _P),
        ("ngroup", ctypes.c_int), ("group_bounds", _P), ("group_list", _P), ("group_param", _P),
        ("group_param_bounds", _P),
    ]


class ValenceUnitView(ctypes.Structure):
    _fields_ = [
        ("imported_atoms", ctypes.c_int), ("moved_atoms", ctypes.c_int),
        ("updated_atoms", ctypes.c_int), ("task_counts", ctypes.c_int * 16),
        ("n_manip", ctypes.c_int),
        ("imports", _P), ("manip", _P), ("update_flags", _P),
        ("bond_terms", _P), ("angl_terms", _P), ("dihe_terms", _P), ("infr14_terms", _P),
        ("cbnd_terms", _P), ("cdhe_terms", _P),
        ("acc_bond", _P), ("acc_angl", _P), ("acc_dihe", _P), ("acc_cbnd", _P),
        ("acc_cdhe", _P), ("acc_infr14", _P),
        ("cbnd_insr", _P), ("angl_insr", _P), ("cdhe_insr", _P), ("infr14_insr", _P),
        ("settle_insr", _P), ("cgroup_insr", _P),
    ]


class Restraint(ctypes.Structure):
    _fields_ = [
        ("system", ctypes.c_int), ("kind", ctypes.c_int), ("atoms", ctypes.c_int * 4),
        ("k2", ctypes.c_double), ("k3", ctypes.c_double), ("r1", ctypes.c_double),
        ("r2", ctypes.c_double), ("r3", ctypes.c_double), ("r4", ctypes.c_double),
        ("target", ctypes.c_double * 3),
        ("init_step", ctypes.c_int), ("final_step", ctypes.c_int),
        ("final_k2", ctypes.c_double), ("final_k3", ctypes.c_double),
        ("final_r1", ctypes.c_double), ("final_r2", ctypes.c_double),
        ("final_r3", ctypes.c_double), ("final_r4", ctypes.c_double),
        ("final_target", ctypes.c_double * 3),
    ]


RESTRAINT_POSITION, RESTRAINT_DISTANCE, RESTRAINT_ANGLE, RESTRAINT_DIHEDRAL = 1, 2, 3, 4


class MinimizeControls(ctypes.Structure):
    _fields_ = [
        ("total_cycles", ctypes.c_int), ("sd_cycles", ctypes.c_int),
        ("clash_cycles", ctypes.c_int), ("initial_step", ctypes.c_double),
        ("convergence_rms", ctypes.c_double), ("record_history", ctypes.c_int),
        ("kernel", ctypes.c_int), ("clash_distance", ctypes.c_double),
        ("clash_ratio", ctypes.c_double),
    ]


class ServerOptions(ctypes.Structure):
    _fields_ = [
        ("options", Options), ("controls", MinimizeControls),
        ("hbm_budget_bytes", ctypes.c_double), ("max_batch_molecules", ctypes.c_int),
        ("max_batches", ctypes.c_int), ("cycles_per_launch", ctypes.c_int),
        ("migrate_fraction", ctypes.c_double),
    ]


class ServedResult(ctypes.Structure):
    _fields_ = [
        ("request_id", ctypes.c_longlong), ("natom", ctypes.c_int), ("kind", ctypes.c_int),
        ("cycles", ctypes.c_int), ("converged", ctypes.c_int), ("status", ctypes.c_int),
        ("rms_force", ctypes.c_double), ("energy", ctypes.c_double),
        ("energies", ctypes.c_double * 16), ("submit_time", ctypes.c_double),
        ("admit_time", ctypes.c_double), ("finish_time", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_longlong), ("admitted", ctypes.c_longlong),
        ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
        ("migrated", ctypes.c_longlong),
        ("pending", ctypes.c_int), ("in_flight", ctypes.c_int),
        ("batches", ctypes.c_int), ("bytes_in_flight", ctypes.c_double),
    ]


class AmberView(ctypes.Structure):
    _fields_ = [
        ("topology", Topology), ("atomic_numbers", _P), ("masses", _P),
        ("exclusion_bounds", _P * 3), ("exclusion_list", _P * 3), ("radius_set", ctypes.c_char_p),
        ("title", ctypes.c_char_p), ("implicit_solvent", ctypes.c_int),
        ("cmap_count", ctypes.c_int), ("urey_bradley_count", ctypes.c_int),
        ("charmm_improper_count", ctypes.c_int), ("unit_cell", ctypes.c_int),
    ]


class SdfView(ctypes.Structure):
    _fields_ = [
        ("title", ctypes.c_char_p), ("natom", ctypes.c_int), ("xyz", ctypes.c_void_p),
        ("atomic_number", ctypes.c_void_p), ("formal_charge", ctypes.c_void_p),
        ("symbols", ctypes.c_void_p), ("nbond", ctypes.c_int), ("bond_i", ctypes.c_void_p),
        ("bond_j", ctypes.c_void_p), ("bond_order", ctypes.c_void_p), ("n_items", ctypes.c_int),
        ("item_names", ctypes.POINTER(ctypes.c_char_p)),
        ("item_contents", ctypes.POINTER(ctypes.c_char_p)),
    ]


class StormmB200Error(RuntimeError):
    pass


_LIB = None


def library() -> ctypes.CDLL:
    """Load libstormm_b200.so; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise StormmB200Error(f"CUDA library not built: {LIB_PATH} "
                                  "(run python -m stormm_b200.build)")
        lib = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "sb_default_options": (None, [ctypes.POINTER(Options)]),
            "sb_synthesis_create": (ctypes.c_int, [ctypes.POINTER(Topology), ctypes.c_int, vp,
                                                   ctypes.c_int, ctypes.POINTER(Options),
                                                   ctypes.POINTER(vp)]),
            "sb_synthesis_destroy": (ctypes.c_int, [vp]),
            "sb_system_count": (ctypes.c_int, [vp]),
            "sb_system_atoms": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int)]),
            "sb_padded_atom_count": (ctypes.c_int, [vp]),
            "sb_set_coordinates": (ctypes.c_int, [vp, vp, vp]),
            "sb_get_coordinates": (ctypes.c_int, [vp, vp, vp]),
            "sb_get_forces": (ctypes.c_int, [vp, vp, vp]),
            "sb_get_energies": (ctypes.c_int, [vp, vp, vp]),
            "sb_download_results_async": (ctypes.c_int, [vp, vp, vp, vp]),
            "sb_set_restraints": (ctypes.c_int, [vp, ctypes.POINTER(Restraint), ctypes.c_int]),
            "sb_set_restraint_step": (ctypes.c_int, [vp, ctypes.c_int]),
            "sb_surface_area": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, vp, vp]),
            "sb_get_gb_workspace": (ctypes.c_int, [vp, vp, vp, vp, vp]),
            "sb_get_forces_fixed": (ctypes.c_int, [vp, vp, vp, vp]),
            "sb_get_energies_fixed": (ctypes.c_int, [vp, vp, vp]),
            "sb_initialize": (ctypes.c_int, [vp, ctypes.c_int, vp]),
            "sb_evaluate": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]),
            "sb_evaluate_range": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, vp]),
            "sb_evaluate_clash": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_double, ctypes.c_double, vp]),
            "sb_launch_nonbonded": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
            "sb_launch_valence": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
            "sb_launch_info": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
            "sb_check_status": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int)]),
            "sb_default_minimize_controls": (None, [ctypes.POINTER(MinimizeControls)]),
            "sb_minimize": (ctypes.c_int, [vp, ctypes.POINTER(MinimizeControls), vp]),
            "sb_minimize_range": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(MinimizeControls), vp]),
            "sb_get_minimize_history": (ctypes.c_int, [vp, vp, vp]),
            "sb_minimize_begin": (ctypes.c_int, [vp, ctypes.POINTER(MinimizeControls), vp]),
            "sb_minimize_advance": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
            "sb_conjugate_gradient": (ctypes.c_int, [vp, vp]),
            "sb_line_advance": (ctypes.c_int, [vp, ctypes.c_int, vp]),
            "sb_autotune": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_double), vp]),
            "sb_get_minimize_progress": (ctypes.c_int, [vp, vp, vp, vp, vp]),
            "sb_default_server_options": (None, [ctypes.POINTER(ServerOptions)]),
            "sb_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOptions),
                                                ctypes.POINTER(vp)]),
            "sb_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(Topology), vp,
                                                ctypes.POINTER(ctypes.c_longlong)]),
            "sb_server_submit_evaluation": (ctypes.c_int, [vp, ctypes.POINTER(Topology), vp,
                                                           ctypes.POINTER(ctypes.c_longlong)]),
            "sb_server_poll": (ctypes.c_int, [vp, ctypes.POINTER(ServedResult), ctypes.c_int, vp,
                                              ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]),
            "sb_server_drain": (ctypes.c_int, [vp, ctypes.c_double]),
            "sb_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
            "sb_server_destroy": (ctypes.c_int, [vp]),
            "sb_static_exclusion_mask": (ctypes.c_int, [ctypes.POINTER(Topology), vp, vp, vp, vp,
                                                        vp, vp, vp]),
            "sb_read_amber_topology": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vp)]),
            "sb_amber_topology_view": (ctypes.c_int, [vp, ctypes.POINTER(AmberView)]),
            "sb_amber_set_implicit_solvent": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
            "sb_amber_topology_destroy": (ctypes.c_int, [vp]),
            "sb_read_amber_coordinates": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, vp]),
            "sb_write_amber_coordinates": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p,
                                                          ctypes.c_int, vp]),
            "sb_read_sdf": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vp)]),
            "sb_sdf_compound_count": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int)]),
            "sb_sdf_compound": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(SdfView)]),
            "sb_sdf_destroy": (ctypes.c_int, [vp]),
            "sb_write_sdf_compound": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int,
                                                     ctypes.POINTER(SdfView)]),
            "sb_static_exclusion_mask_synthesis": (ctypes.c_int, [ctypes.POINTER(Topology),
                                                                  ctypes.c_int, vp, ctypes.c_int,
                                                                  vp, vp, vp, vp, vp, vp, vp]),
            "sb_nonbonded_work_units": (ctypes.c_int, [ctypes.POINTER(Topology), ctypes.c_int, vp,
                                                       ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                       vp, vp, vp, vp]),
            "sb_valence_work_units": (ctypes.c_int, [ctypes.POINTER(ValenceTopology),
                                                     ctypes.c_int, ctypes.c_int,
                                                     ctypes.POINTER(vp)]),
            "sb_valence_units_destroy": (ctypes.c_int, [vp]),
            "sb_valence_unit_count": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int)]),
            "sb_valence_unit": (ctypes.c_int, [vp, ctypes.c_int,
                                               ctypes.POINTER(ValenceUnitView)]),
            "sb_valence_work_unit_size": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_int),
                                                         ctypes.POINTER(ctypes.c_int)]),
            "sb_last_error": (ctypes.c_char_p, []),
            "sb_version": (ctypes.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _check(rc: int, what: str) -> None:
    if rc != SB_OK:
        msg = library().sb_last_error().decode(errors="replace")
        raise StormmB200Error(f"{what} failed ({rc}): {msg}")


def default_options(**overrides) -> Options:
    """sb_default_options with overrides by field name.  The neck GB tables
    (neck_max_separation, neck_max_value) may be given as arrays; the returned Options keeps
    them alive (sb_synthesis_create copies them)."""
    o = Options()
    library().sb_default_options(ctypes.byref(o))
    keep = []
    for k, v in overrides.items():
        if k in ("neck_max_separation", "neck_max_value") and v is not None and \
                not isinstance(v, int):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1))
            keep.append(a)
            v = a.ctypes.data
        setattr(o, k, v)
    o._keep = keep
    return o


class _TopologyArrays:
    """Keeps the numpy arrays behind one sb_topology alive."""

    def __init__(self, mol):
        self.keep = []
        t = Topology()

        def ptr(a, dt):
            a = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dt)
            self.keep.append(a)
            return a.ctypes.data

        n = mol.natom
        t.natom = n
        t.charge = ptr(mol.charge, np.float64)
        t.lj_idx = ptr(mol.lj_idx, np.int32)
        t.n_lj_types = mol.n_lj_types
        t.lja = ptr(mol.lja, np.float64)
        t.ljb = ptr(mol.ljb, np.float64)
        lja14 = getattr(mol, "lja14", None)
        ljb14 = getattr(mol, "ljb14", None)
        t.lja14 = ptr(lja14, np.float64) if lja14 is not None else None
        t.ljb14 = ptr(ljb14, np.float64) if ljb14 is not None else None
        bounds = np.zeros(n + 1, dtype=np.int32)
        items = []
        for i in range(n):
            part = sorted(set(mol.excl12[i]) | set(mol.excl13[i]) | set(mol.excl14[i]))
            items.extend(part)
            bounds[i + 1] = len(items)
        t.excl_bounds = ptr(bounds, np.int32)
        t.excl_list = ptr(np.array(items if items else [0], dtype=np.int32), np.int32)
        t.pb_radii = ptr(mol.pb_radii, np.float64)
        t.gb_screen = ptr(mol.gb_screen, np.float64)
        for name in ("gb_alpha", "gb_beta", "gb_gamma"):
            v = getattr(mol, name, None)
            setattr(t, name, ptr(v, np.float64) if v is not None else None)
        t.nbond = mol.bonds.shape[0]
        t.bond_atoms = ptr(mol.bonds, np.int32)
        t.bond_keq = ptr(mol.bond_k, np.float64)
        t.bond_leq = ptr(mol.bond_r0, np.float64)
        t.nangl = mol.angles.shape[0]
        t.angl_atoms = ptr(mol.angles, np.int32)
        t.angl_keq = ptr(mol.angl_k, np.float64)
        t.angl_theta0 = ptr(mol.angl_theta0, np.float64)
        t.ndihe = mol.dihedrals.shape[0]
        t.dihe_atoms = ptr(mol.dihedrals, np.int32)
        t.dihe_amp = ptr(mol.dihe_amp, np.float64)
        t.dihe_freq = ptr(mol.dihe_freq, np.float64)
        t.dihe_phase = ptr(mol.dihe_phase, np.float64)
        scee = getattr(mol, "dihe_scee_array", None)
        scnb = getattr(mol, "dihe_scnb_array", None)
        has14 = np.asarray(mol.dihe_has14, dtype=bool)
        if scee is None:
            scee = np.where(has14, mol.scee, 0.0)
        if scnb is None:
            scnb = np.where(has14, mol.scnb, 0.0)
        t.dihe_scee = ptr(scee, np.float64)
        t.dihe_scnb = ptr(scnb, np.float64)
        impr = getattr(mol, "dihe_improper", None)
        t.dihe_improper = ptr(impr, np.int32) if impr is not None else None
        # CHARMM terms, when the molecule carries them
        ub = getattr(mol, "ubrd_atoms", None)
        if ub is not None and len(ub) > 0:
            t.nubrd = len(np.asarray(ub).reshape(-1, 2))
            t.ubrd_atoms = ptr(ub, np.int32)
            t.ubrd_keq = ptr(mol.ubrd_keq, np.float64)
            t.ubrd_leq = ptr(mol.ubrd_leq, np.float64)
        ci = getattr(mol, "cimp_atoms", None)
        if ci is not None and len(ci) > 0:
            t.ncimp = len(np.asarray(ci).reshape(-1, 4))
            t.cimp_atoms = ptr(ci, np.int32)
            t.cimp_keq = ptr(mol.cimp_keq, np.float64)
            t.cimp_phase = ptr(mol.cimp_phase, np.float64)
        cm = getattr(mol, "cmap_atoms", None)
        if cm is not None and len(cm) > 0:
            t.ncmap = len(np.asarray(cm).reshape(-1, 5))
            t.cmap_atoms = ptr(cm, np.int32)
            t.cmap_surface = ptr(mol.cmap_surface, np.int32)
            t.ncmap_surf = len(mol.cmap_dims)
            t.cmap_dims = ptr(mol.cmap_dims, np.int32)
            t.cmap_values = ptr(mol.cmap_values, np.float64)
        self.struct = t


def static_exclusion_mask(molecule):
    """STORMM's StaticExclusionMask tables of one molecule (host only): a dict with
    supertile_stride_count, supertile_map_idx, tile_map_idx and mask_data."""
    lib = library()
    t = _TopologyArrays(molecule)
    nst = ctypes.c_int()
    n = [ctypes.c_longlong(0) for _ in range(3)]
    _check(lib.sb_static_exclusion_mask(ctypes.byref(t.struct), ctypes.byref(nst), None,
                                        ctypes.byref(n[0]), None, ctypes.byref(n[1]), None,
                                        ctypes.byref(n[2])), "sb_static_exclusion_mask")
    sup = np.zeros(n[0].value, dtype=np.int32)
    til = np.zeros(n[1].value, dtype=np.int32)
    msk = np.zeros(n[2].value, dtype=np.uint32)
    _check(lib.sb_static_exclusion_mask(ctypes.byref(t.struct), ctypes.byref(nst),
                                        sup.ctypes.data, ctypes.byref(n[0]), til.ctypes.data,
                                        ctypes.byref(n[1]), msk.ctypes.data,
                                        ctypes.byref(n[2])), "sb_static_exclusion_mask")
    return {"supertile_stride_count": nst.value, "supertile_map_idx": sup,
            "tile_map_idx": til, "mask_data": msk}


def _synthesis_topologies(molecules, topology_index):
    mols = list(molecules)
    if topology_index is None:
        topology_index = np.arange(len(mols), dtype=np.int32)
    index = np.ascontiguousarray(topology_index, dtype=np.int32)
    tops = [_TopologyArrays(m) for m in mols]
    arr = (Topology * len(mols))(*[t.struct for t in tops])
    return tops, arr, index


def static_exclusion_mask_synthesis(molecules, topology_index=None):
    """STORMM's StaticExclusionMaskSynthesis tables (host only): a dict with
    supertile_map_bounds, supertile_map_idx, tile_map_idx and mask_data."""
    lib = library()
    tops, arr, index = _synthesis_topologies(molecules, topology_index)
    bounds = np.zeros(index.size + 1, dtype=np.int32)
    n = [ctypes.c_longlong(0) for _ in range(3)]
    args = (arr, len(tops), index.ctypes.data, index.size)
    _check(lib.sb_static_exclusion_mask_synthesis(*args, None, None, ctypes.byref(n[0]), None,
                                                  ctypes.byref(n[1]), None, ctypes.byref(n[2])),
           "sb_static_exclusion_mask_synthesis")
    sup = np.zeros(n[0].value, dtype=np.int32)
    til = np.zeros(n[1].value, dtype=np.int32)
    msk = np.zeros(n[2].value, dtype=np.uint32)
    _check(lib.sb_static_exclusion_mask_synthesis(*args, bounds.ctypes.data, sup.ctypes.data,
                                                  ctypes.byref(n[0]), til.ctypes.data,
                                                  ctypes.byref(n[1]), msk.ctypes.data,
                                                  ctypes.byref(n[2])),
           "sb_static_exclusion_mask_synthesis")
    return {"supertile_map_bounds": bounds, "supertile_map_idx": sup, "tile_map_idx": til,
            "mask_data": msk}


def nonbonded_work_units(molecules, topology_index=None, init_task=3, random_cache_depth=0):
    """STORMM's nonbonded work units for a synthesis (host only): (abstracts as an
    (n_units, 64) int32 array, tile instructions as an (n, 2) uint32 array).  init_task is
    STORMM's InitializationTask (3 = GB_MINIMIZATION)."""
    lib = library()
    tops, arr, index = _synthesis_topologies(molecules, topology_index)
    na, ni = ctypes.c_longlong(0), ctypes.c_longlong(0)
    args = (arr, len(tops), index.ctypes.data, index.size, int(init_task),
            int(random_cache_depth))
    _check(lib.sb_nonbonded_work_units(*args, None, ctypes.byref(na), None, ctypes.byref(ni)),
           "sb_nonbonded_work_units")
    a = np.zeros(na.value, dtype=np.int32)
    ins = np.zeros(ni.value, dtype=np.uint32)
    _check(lib.sb_nonbonded_work_units(*args, a.ctypes.data, ctypes.byref(na), ins.ctypes.data,
                                       ctypes.byref(ni)), "sb_nonbonded_work_units")
    return a.reshape(-1, 64), ins.reshape(-1, 2)


_VWU_COUNTS = {"bond": "nbond", "angl": "nangl", "dihe": "ndihe", "infr14": "ninfr14",
               "settle": "nsettle"}


def valence_work_units(top, atom_limit, solvent_atom_limit=None):
    """STORMM's valence work units of one topology (host only), from a dict of its ValenceKit /
    ConstraintKit / NonbondedKit arrays in STORMM's order (keys as the fields of
    sb_valence_topology; a missing optional array is NULL).  Returns one dict per unit: counts,
    imports, manipulation masks ((n, 2) uint32), task counts (VWU_TASKS order), term lists,
    energy-accumulation masks and instructions ((n, words) uint32)."""
    lib = library()
    keep = []

    def arr(key, dtype=np.int32):
        v = top.get(key)
        if v is None:
            return None
        a = np.ascontiguousarray(np.asarray(v), dtype=dtype)
        keep.append(a)
        return a.ctypes.data

    t = ValenceTopology()
    t.natom = int(top["natom"])
    for f, _ in ValenceTopology._fields_:
        if f == "natom":
            continue
        if f.startswith("n") and f not in ("nb12_bounds", "nb12_list"):
            continue
        setattr(t, f, arr(f, np.uint32 if f.endswith("relevance") else np.int32))
    for stem, count in _VWU_COUNTS.items():
        first = {"bond": "bond_i", "angl": "angl_i", "dihe": "dihe_i", "infr14": "infr14_i",
                 "settle": "settle_ox"}[stem]
        setattr(t, count, 0 if top.get(first) is None else len(top[first]))
    t.ngroup = 0 if top.get("group_bounds") is None else len(top["group_bounds"]) - 1
    h = ctypes.c_void_p()
    lim = int(atom_limit)
    slim = lim if solvent_atom_limit is None else int(solvent_atom_limit)
    _check(lib.sb_valence_work_units(ctypes.byref(t), lim, slim, ctypes.byref(h)),
           "sb_valence_work_units")
    try:
        n = ctypes.c_int()
        _check(lib.sb_valence_unit_count(h, ctypes.byref(n)), "sb_valence_unit_count")
        out = []
        for k in range(n.value):
            v = ValenceUnitView()
            _check(lib.sb_valence_unit(h, k, ctypes.byref(v)), "sb_valence_unit")
            tc = list(v.task_counts)
            u32 = lambda p, c: _host_array(p, c, ctypes.c_uint32, np.uint32)
            i32 = lambda p, c: _host_array(p, c, ctypes.c_int, np.int32)
            words = lambda c: (c + 31) // 32
            nb, na, nd, ncb, ncd, nin, nst, ncg = (tc[0], tc[1], tc[2], tc[4], tc[6], tc[8],
                                                   tc[14], tc[15])
            out.append({
                "imported": v.imported_atoms, "moved": v.moved_atoms, "updated": v.updated_atoms,
                "task_counts": np.array(tc, dtype=np.int32),
                "imports": i32(v.imports, v.imported_atoms),
                "manip": u32(v.manip, 2 * v.n_manip).reshape(-1, 2),
                "update_flags": u32(v.update_flags, words(v.imported_atoms)),
                "bond_terms": i32(v.bond_terms, nb), "angl_terms": i32(v.angl_terms, na),
                "dihe_terms": i32(v.dihe_terms, nd), "infr14_terms": i32(v.infr14_terms, nin),
                "cbnd_terms": i32(v.cbnd_terms, ncb),
                "cdhe_terms": i32(v.cdhe_terms, 2 * ncd).reshape(-1, 2),
                "acc_bond": u32(v.acc_bond, words(nb)), "acc_angl": u32(v.acc_angl, words(na)),
                "acc_dihe": u32(v.acc_dihe, words(nd)), "acc_cbnd": u32(v.acc_cbnd, words(ncb)),
                "acc_cdhe": u32(v.acc_cdhe, words(ncd)),
                "acc_infr14": u32(v.acc_infr14, words(nin)),
                "cbnd_insr": u32(v.cbnd_insr, 2 * ncb).reshape(-1, 2),
                "angl_insr": u32(v.angl_insr, 2 * na).reshape(-1, 2),
                "cdhe_insr": u32(v.cdhe_insr, 3 * ncd).reshape(-1, 3),
                "infr14_insr": u32(v.infr14_insr, nin),
                "settle_insr": u32(v.settle_insr, 2 * nst).reshape(-1, 2),
                "cgroup_insr": u32(v.cgroup_insr, 2 * ncg).reshape(-1, 2),
            })
        return out
    finally:
        lib.sb_valence_units_destroy(h)


def valence_work_unit_size(atom_counts, sm_count):
    """STORMM's calculateValenceWorkUnitSize for isolated systems: (atom limit, kernel width
    0-3 = XL/LG/MD/SM, or None without an SM count)."""
    c = np.ascontiguousarray(atom_counts, dtype=np.int32)
    lim, width = ctypes.c_int(), ctypes.c_int(-1)
    _check(library().sb_valence_work_unit_size(c.ctypes.data, c.size, int(sm_count),
                                                ctypes.byref(lim), ctypes.byref(width)),
           "sb_valence_work_unit_size")
    return lim.value, (width.value if sm_count > 0 else None)


def _host_array(ptr, count, ctype, dtype):
    """Copy of count values at a library-owned pointer (empty when count is 0)."""
    if count == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)),
                                 shape=(count,)).astype(dtype, copy=True)


def read_amber(prmtop, inpcrd=None, igb=None, radius_set=0):
    """A molecule from an Amber topology file and, optionally, its coordinate file: what
    STORMM's AtomGraph(file_name) and PhaseSpace(file_name) read (Topology/atomgraph.h:83,156).
    With igb, the per-atom GB parameters of that model are assigned as STORMM's
    AtomGraph::setImplicitSolventModel assigns them: radius_set (RADII_*, default the file's
    radii) first, then element screening factors for the neck models.  Returns a synthetic.Molecule (coordinates zero without inpcrd) carrying, besides
    the usual fields, the per-dihedral 1-4 factors, improper flags, the 1-4 Lennard-Jones
    tables when the file has them, the GB parameters when igb is given, and the file's title,
    radius set and CHARMM term counts."""
    from .synthetic import Molecule
    lib = library()
    h = ctypes.c_void_p()
    _check(lib.sb_read_amber_topology(os.fsencode(str(prmtop)), ctypes.byref(h)),
           "sb_read_amber_topology")
    try:
        if igb is not None:
            _check(lib.sb_amber_set_implicit_solvent(h, int(igb), int(radius_set)),
                   "sb_amber_set_implicit_solvent")
        v = AmberView()
        _check(lib.sb_amber_topology_view(h, ctypes.byref(v)), "sb_amber_topology_view")
        t = v.topology
        n, nt = t.natom, t.n_lj_types
        dbl, i32 = ctypes.c_double, ctypes.c_int

        def d(p, c):
            return _host_array(p, c, dbl, np.float64)

        def i(p, c):
            return _host_array(p, c, i32, np.int32)

        excl = []
        for lv in range(3):
            b = i(v.exclusion_bounds[lv], n + 1)
            x = i(v.exclusion_list[lv], int(b[-1]))
            excl.append([list(x[b[a]:b[a + 1]]) for a in range(n)])
        scee = d(t.dihe_scee, t.ndihe)
        mol = Molecule(
            natom=n, coords=np.zeros((n, 3)), charge=d(t.charge, n), lj_idx=i(t.lj_idx, n),
            lja=d(t.lja, nt * nt).reshape(nt, nt), ljb=d(t.ljb, nt * nt).reshape(nt, nt),
            z_numbers=i(v.atomic_numbers, n), mass=d(v.masses, n), pb_radii=d(t.pb_radii, n),
            gb_screen=d(t.gb_screen, n), bonds=i(t.bond_atoms, 2 * t.nbond).reshape(-1, 2),
            bond_k=d(t.bond_keq, t.nbond), bond_r0=d(t.bond_leq, t.nbond),
            angles=i(t.angl_atoms, 3 * t.nangl).reshape(-1, 3),
            angl_k=d(t.angl_keq, t.nangl), angl_theta0=d(t.angl_theta0, t.nangl),
            dihedrals=i(t.dihe_atoms, 4 * t.ndihe).reshape(-1, 4),
            dihe_amp=d(t.dihe_amp, t.ndihe), dihe_freq=d(t.dihe_freq, t.ndihe),
            dihe_phase=d(t.dihe_phase, t.ndihe), dihe_has14=scee > 0.0,
            name=(v.title or b"").decode(errors="replace").strip() or "MOL",
            excl12=excl[0], excl13=excl[1], excl14=excl[2])
        mol.dihe_scee_array = scee
        mol.dihe_scnb_array = d(t.dihe_scnb, t.ndihe)
        mol.dihe_improper = i(t.dihe_improper, t.ndihe)
        if t.lja14:
            mol.lja14 = d(t.lja14, nt * nt).reshape(nt, nt)
            mol.ljb14 = d(t.ljb14, nt * nt).reshape(nt, nt)
        if igb is not None:
            mol.gb_alpha = d(t.gb_alpha, n)
            mol.gb_beta = d(t.gb_beta, n)
            mol.gb_gamma = d(t.gb_gamma, n)
        mol.radius_set = (v.radius_set or b"").decode(errors="replace")
        mol.cmap_count = v.cmap_count
        mol.urey_bradley_count = v.urey_bradley_count
        mol.charmm_improper_count = v.charmm_improper_count
        if t.nubrd > 0:
            mol.ubrd_atoms = i(t.ubrd_atoms, 2 * t.nubrd).reshape(-1, 2)
            mol.ubrd_keq = d(t.ubrd_keq, t.nubrd)
            mol.ubrd_leq = d(t.ubrd_leq, t.nubrd)
        if t.ncimp > 0:
            mol.cimp_atoms = i(t.cimp_atoms, 4 * t.ncimp).reshape(-1, 4)
            mol.cimp_keq = d(t.cimp_keq, t.ncimp)
            mol.cimp_phase = d(t.cimp_phase, t.ncimp)
        if t.ncmap > 0:
            mol.cmap_atoms = i(t.cmap_atoms, 5 * t.ncmap).reshape(-1, 5)
            mol.cmap_surface = i(t.cmap_surface, t.ncmap)
            mol.cmap_dims = i(t.cmap_dims, t.ncmap_surf)
            mol.cmap_values = d(t.cmap_values, int((mol.cmap_dims.astype(np.int64) ** 2).sum()))
        mol.unit_cell = v.unit_cell
    finally:
        lib.sb_amber_topology_destroy(h)
    if inpcrd is not None:
        mol.coords = read_amber_coordinates(inpcrd, mol.natom)
    return mol


def read_amber_coordinates(path, natom):
    """(natom, 3) coordinates of an Amber ASCII coordinate / restart file."""
    xyz = np.zeros(3 * natom)
    _check(library().sb_read_amber_coordinates(os.fsencode(str(path)), int(natom),
                                               xyz.ctypes.data), "sb_read_amber_coordinates")
    return xyz.reshape(natom, 3)


def write_amber_coordinates(path, xyz, title=""):
    """Write (natom, 3) coordinates as an Amber input-coordinate file (STORMM's AMBER_INPCRD)."""
    c = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1))
    _check(library().sb_write_amber_coordinates(os.fsencode(str(path)), title.encode(),
                                                c.size // 3, c.ctypes.data),
           "sb_write_amber_coordinates")


def read_sdf(path):
    """Compounds of an SD / MOL file (V2000) as dicts: title, xyz (natom, 3), atomic_number,
    formal_charge, symbols, bonds (nbond, 3: i, j, MDL type), items {name: text}."""
    lib = library()
    h = ctypes.c_void_p()
    _check(lib.sb_read_sdf(os.fsencode(str(path)), ctypes.byref(h)), "sb_read_sdf")
    try:
        n = ctypes.c_int()
        _check(lib.sb_sdf_compound_count(h, ctypes.byref(n)), "sb_sdf_compound_count")
        out = []
        for k in range(n.value):
            v = SdfView()
            _check(lib.sb_sdf_compound(h, k, ctypes.byref(v)), "sb_sdf_compound")
            na, nb = v.natom, v.nbond

            def arr(ptr, count, ct, dt):
                if count == 0 or not ptr:
                    return np.zeros(0, dtype=dt)
                return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)),
                                             shape=(count,)).astype(dt)
            sym = ctypes.string_at(v.symbols, 4 * na)
            bonds = np.stack([arr(v.bond_i, nb, ctypes.c_int, np.int32),
                              arr(v.bond_j, nb, ctypes.c_int, np.int32),
                              arr(v.bond_order, nb, ctypes.c_int, np.int32)], axis=1)
            out.append({
                "title": v.title.decode(errors="replace"),
                "xyz": arr(v.xyz, 3 * na, ctypes.c_double, np.float64).reshape(na, 3),
                "atomic_number": arr(v.atomic_number, na, ctypes.c_int, np.int32),
                "formal_charge": arr(v.formal_charge, na, ctypes.c_int, np.int32),
                "symbols": [sym[4 * a:4 * a + 4].rstrip(b"\0").decode() for a in range(na)],
                "bonds": bonds,
                "items": {v.item_names[i].decode(): v.item_contents[i].decode()
                          for i in range(v.n_items)},
            })
        return out
    finally:
        lib.sb_sdf_destroy(h)


def write_sdf(path, compound, append=False):
    """Write one compound (a dict as read_sdf returns; symbols or atomic_number, optional
    formal_charge, bonds and items) as a V2000 SD entry."""
    na = len(compound["xyz"])
    xyz = np.ascontiguousarray(np.asarray(compound["xyz"], dtype=np.float64).reshape(-1))
    keep = [xyz]
    v = SdfView()
    v.title = compound.get("title", "").encode()
    v.natom = na
    v.xyz = xyz.ctypes.data
    if compound.get("symbols") is not None:
        buf = ctypes.create_string_buffer(b"".join(s.encode()[:3].ljust(4, b"\0")
                                                   for s in compound["symbols"]), 4 * na)
        keep.append(buf)
        v.symbols = ctypes.addressof(buf)
    if compound.get("atomic_number") is not None:
        z = np.ascontiguousarray(compound["atomic_number"], dtype=np.int32)
        keep.append(z)
        v.atomic_number = z.ctypes.data
    if compound.get("formal_charge") is not None:
        q = np.ascontiguousarray(compound["formal_charge"], dtype=np.int32)
        keep.append(q)
        v.formal_charge = q.ctypes.data
    bonds = np.asarray(compound.get("bonds", np.zeros((0, 3))), dtype=np.int32).reshape(-1, 3)
    v.nbond = len(bonds)
    cols = [np.ascontiguousarray(bonds[:, c]) for c in range(3)]
    keep.extend(cols)
    if len(bonds):
        v.bond_i, v.bond_j, v.bond_order = (c.ctypes.data for c in cols)
    items = compound.get("items", {})
    names = (ctypes.c_char_p * max(1, len(items)))(*[k.encode() for k in items])
    texts = (ctypes.c_char_p * max(1, len(items)))(*[t.encode() for t in items.values()])
    v.n_items = len(items)
    v.item_names = names
    v.item_contents = texts
    _check(library().sb_write_sdf_compound(os.fsencode(str(path)), int(bool(append)),
                                           ctypes.byref(v)), "sb_write_sdf_compound")


def minimize_controls(**overrides) -> MinimizeControls:
    """STORMM's minimizer defaults (maxcyc 200, ncyc 50, dx0 0.01; no clash-damped cycles,
    softened cores of 0.2 A and 0.5 sigma when clash_cycles is set) with overrides by field
    name."""
    c = MinimizeControls()
    library().sb_default_minimize_controls(ctypes.byref(c))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


class Synthesis:
    """A batch of molecules resident on the GPU (STORMM's AtomGraphSynthesis +
    PhaseSpaceSynthesis + ImplicitSolventWorkspace + ScoreCard for this path)."""

    def __init__(self, molecules, topology_index=None, options: Options | None = None, **opts):
        lib = library()
        mols = list(molecules)
        if topology_index is None:
            topology_index = np.arange(len(mols), dtype=np.int32)
        self.topology_index = np.ascontiguousarray(topology_index, dtype=np.int32)
        self._tops = [_TopologyArrays(m) for m in mols]
        arr = (Topology * len(mols))(*[t.struct for t in self._tops])
        o = options if options is not None else default_options(**opts)
        handle = ctypes.c_void_p()
        _check(lib.sb_synthesis_create(arr, len(mols), self.topology_index.ctypes.data,
                                       len(self.topology_index), ctypes.byref(o),
                                       ctypes.byref(handle)), "sb_synthesis_create")
        self.handle = handle
        self.nsys = len(self.topology_index)
        self.natoms = np.array([mols[t].natom for t in self.topology_index], dtype=np.int64)
        self.total_atoms = int(self.natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)])

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            library().sb_synthesis_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # transfers -----------------------------------------------------------------------------
    def set_coordinates(self, xyz, stream=None):
        a = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1))
        if a.size != 3 * self.total_atoms:
            raise ValueError("coordinate array does not match the synthesis atom count")
        _check(library().sb_set_coordinates(self.handle, a.ctypes.data, stream),
               "sb_set_coordinates")

    @staticmethod
    def _output(out, n):
        """A float64 buffer of n values: a new array, or the caller's (reused, e.g. pinned)."""
        if out is None:
            return np.zeros(n)
        if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.size != n or
                not out.flags["C_CONTIGUOUS"]):
            raise ValueError(f"output buffer must be a contiguous float64 array of {n} values")
        return out

    def coordinates(self, stream=None, out=None):
        out = self._output(out, 3 * self.total_atoms)
        _check(library().sb_get_coordinates(self.handle, out.ctypes.data, stream),
               "sb_get_coordinates")
        return out.reshape(-1, 3)

    def forces(self, stream=None, out=None):
        """Forces (kcal/mol/A, unpadded atoms); `out` may be a reused (pinned) buffer."""
        out = self._output(out, 3 * self.total_atoms)
        _check(library().sb_get_forces(self.handle, out.ctypes.data, stream), "sb_get_forces")
        return out.reshape(-1, 3)

    def energies(self, stream=None, out=None):
        out = self._output(out, self.nsys * NRG_STRIDE)
        _check(library().sb_get_energies(self.handle, out.ctypes.data, stream),
               "sb_get_energies")
        return out.reshape(self.nsys, NRG_STRIDE)

    def set_restraints(self, restraints):
        """Replace the synthesis's restraints: an iterable of dicts with system, kind
        (RESTRAINT_*), atoms, k2, k3, r1-r4 and, for positional ones, target; a time-dependent
        restraint adds init_step, final_step and the final_* values (the same names with a
        final_ prefix), which it reaches by a linear ramp between the two steps."""
        rs = list(restraints)
        arr = (Restraint * max(1, len(rs)))()
        for q, r in enumerate(rs):
            a = list(r["atoms"]) + [0] * (4 - len(r["atoms"]))
            arr[q].system = int(r.get("system", 0))
            arr[q].kind = int(r["kind"])
            for m in range(4):
                arr[q].atoms[m] = int(a[m])
            for f in ("k2", "k3", "r1", "r2", "r3", "r4"):
                setattr(arr[q], f, float(r[f]))
            t = r.get("target", (0.0, 0.0, 0.0))
            for m in range(3):
                arr[q].target[m] = float(t[m])
            arr[q].init_step = int(r.get("init_step", 0))
            arr[q].final_step = int(r.get("final_step", arr[q].init_step))
            for f in ("k2", "k3", "r1", "r2", "r3", "r4"):
                setattr(arr[q], "final_" + f, float(r.get("final_" + f, 0.0)))
            t = r.get("final_target", (0.0, 0.0, 0.0))
            for m in range(3):
                arr[q].final_target[m] = float(t[m])
        _check(library().sb_set_restraints(self.handle, arr, len(rs)), "sb_set_restraints")

    def surface_area(self, sphere_points, probe_radius=1.4, weight=1.0, stream=None):
        """STORMM's sphere-point surface area of every system (sb_surface_area): sphere_points
        is an (n, 3) array of unit vectors; weight 1 gives A^2, 0.005 STORMM's default energy
        in kcal/mol."""
        pts = np.ascontiguousarray(sphere_points, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(self.nsys)
        _check(library().sb_surface_area(self.handle, pts.ctypes.data, len(pts),
                                         float(probe_radius), float(weight), out.ctypes.data,
                                         stream), "sb_surface_area")
        return out

    def set_restraint_step(self, step):
        """The step at which evaluations take time-dependent restraints (sb_set_restraint_step;
        the graph minimizer uses each system's cycle count instead)."""
        _check(library().sb_set_restraint_step(self.handle, int(step)), "sb_set_restraint_step")

    def download_async(self, forces=None, energies=None, stream=None):
        """Enqueue the forces (3 per atom) and energies (nsys x NRG_STRIDE) into page-locked
        float64 buffers on the stream without waiting (sb_download_results_async)."""
        f = None if forces is None else self._output(forces, 3 * self.total_atoms)
        e = None if energies is None else self._output(energies, self.nsys * NRG_STRIDE)
        _check(library().sb_download_results_async(
            self.handle, None if f is None else f.ctypes.data,
            None if e is None else e.ctypes.data, stream), "sb_download_results_async")

    def energy_terms(self, stream=None):
        """Per system, the nine terms in TERM_ORDER."""
        e = self.energies(stream)
        return e[:, [NRG_SLOTS[n] for n in TERM_ORDER]]

    def gb_workspace(self, stream=None):
        psi = np.zeros(self.total_atoms)
        rad = np.zeros(self.total_atoms)
        sde = np.zeros(self.total_atoms)
        _check(library().sb_get_gb_workspace(self.handle, psi.ctypes.data, rad.ctypes.data,
                                             sde.ctypes.data, stream), "sb_get_gb_workspace")
        return psi, rad, sde

    def forces_fixed(self, stream=None):
        n = library().sb_padded_atom_count(self.handle)
        prim = np.zeros(3 * n, dtype=np.int64)
        ovrf = np.zeros(3 * n, dtype=np.int32)
        _check(library().sb_get_forces_fixed(self.handle, prim.ctypes.data, ovrf.ctypes.data,
                                             stream), "sb_get_forces_fixed")
        return prim.reshape(3, n), ovrf.reshape(3, n)

    def energies_fixed(self, stream=None):
        out = np.zeros(self.nsys * NRG_STRIDE, dtype=np.int64)
        _check(library().sb_get_energies_fixed(self.handle, out.ctypes.data, stream),
               "sb_get_energies_fixed")
        return out.reshape(self.nsys, NRG_STRIDE)

    # evaluation ----------------------------------------------------------------------------
    def initialize(self, what=INIT_FORCES | INIT_ENERGIES | INIT_GB_WORKSPACE, stream=None):
        _check(library().sb_initialize(self.handle, what, stream), "sb_initialize")

    def evaluate(self, terms=TERM_ALL, force=True, energy=True, stream=None):
        _check(library().sb_evaluate(self.handle, terms, int(force), int(energy), stream),
               "sb_evaluate")

    def evaluate_range(self, first, count, terms=TERM_ALL, force=True, energy=True,
                       stream=None):
        _check(library().sb_evaluate_range(self.handle, first, count, terms, int(force),
                                           int(energy), stream), "sb_evaluate_range")

    def evaluate_clash(self, clash_distance, clash_ratio, terms=TERM_ALL, force=True,
                       energy=True, stream=None):
        """evaluate() with softened Coulomb / Lennard-Jones cores (sb_evaluate_clash)."""
        _check(library().sb_evaluate_clash(self.handle, terms, int(force), int(energy),
                                           float(clash_distance), float(clash_ratio), stream),
               "sb_evaluate_clash")

    def launch_nonbonded(self, force=True, energy=True, stream=None):
        _check(library().sb_launch_nonbonded(self.handle, int(force), int(energy), stream),
               "sb_launch_nonbonded")

    def launch_valence(self, force=True, energy=True, stream=None):
        _check(library().sb_launch_valence(self.handle, int(force), int(energy), stream),
               "sb_launch_valence")

    # minimization ------------------------------------------------------------------------
    def minimize(self, stream=None, **controls):
        """Line-minimize every system in place (fields of MinimizeControls as keywords)."""
        c = minimize_controls(**controls)
        self._history_stride = c.total_cycles + 1 if c.record_history else 0
        _check(library().sb_minimize(self.handle, ctypes.byref(c), stream), "sb_minimize")

    def minimize_begin(self, stream=None, **controls):
        """Reset every system's minimizer state (sb_minimize_begin)."""
        c = minimize_controls(**controls)
        self._history_stride = c.total_cycles + 1 if c.record_history else 0
        _check(library().sb_minimize_begin(self.handle, ctypes.byref(c), stream),
               "sb_minimize_begin")

    def minimize_advance(self, cycles, final_energy=True, stream=None):
        """Run up to `cycles` more cycles of every unfinished system (sb_minimize_advance)."""
        _check(library().sb_minimize_advance(self.handle, int(cycles), int(final_energy), stream),
               "sb_minimize_advance")

    def conjugate_gradient(self, stream=None):
        """One conjugate-gradient step of every system (sb_conjugate_gradient)."""
        _check(library().sb_conjugate_gradient(self.handle, stream), "sb_conjugate_gradient")

    def line_advance(self, move_number, stream=None):
        """One line-search move 0-3 of every active system (sb_line_advance)."""
        _check(library().sb_line_advance(self.handle, int(move_number), stream),
               "sb_line_advance")

    def autotune(self, what=TUNE_EVALUATE, stream=None):
        """Pick the fastest work-unit packing; returns (atoms per unit, tiles per unit, ms)."""
        a, t, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(library().sb_autotune(self.handle, what, ctypes.byref(a), ctypes.byref(t),
                                     ctypes.byref(ms), stream), "sb_autotune")
        return a.value, t.value, ms.value

    def minimize_range(self, first, count, stream=None, **controls):
        """The same with one launch per system, systems [first, first + count)."""
        c = minimize_controls(**controls)
        self._history_stride = c.total_cycles + 1 if c.record_history else 0
        _check(library().sb_minimize_range(self.handle, first, count, ctypes.byref(c), stream),
               "sb_minimize_range")

    def minimize_history(self, stream=None):
        """(nsys, total_cycles + 1) energies of the last minimization run with history."""
        stride = getattr(self, "_history_stride", 0)
        if stride == 0:
            raise StormmB200Error("the last minimization kept no history")
        out = np.zeros(self.nsys * stride)
        _check(library().sb_get_minimize_history(self.handle, out.ctypes.data, stream),
               "sb_get_minimize_history")
        return out.reshape(self.nsys, stride)

    def minimize_progress(self, stream=None):
        """(cycles completed, converged flags, latest RMS force) per system."""
        cyc = np.zeros(self.nsys, dtype=np.int32)
        conv = np.zeros(self.nsys, dtype=np.int32)
        rms = np.zeros(self.nsys)
        _check(library().sb_get_minimize_progress(self.handle, cyc.ctypes.data, conv.ctypes.data,
                                                  rms.ctypes.data, stream),
               "sb_get_minimize_progress")
        return cyc, conv.astype(bool), rms

    def launch_info(self):
        u, b, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(library().sb_launch_info(self.handle, ctypes.byref(u), ctypes.byref(b),
                                        ctypes.byref(t)), "sb_launch_info")
        return {"work_units": u.value, "blocks": b.value, "threads": t.value}

    def status(self):
        st = ctypes.c_int()
        _check(library().sb_check_status(self.handle, ctypes.byref(st)), "sb_check_status")
        return st.value

    def split(self, per_atom):
        """Split a per-atom array of the whole synthesis into per-system arrays."""
        return [per_atom[self.offsets[k]:self.offsets[k + 1]] for k in range(self.nsys)]


SB_TIMEOUT = 1


class Server:
    """Continuous-batching request server (sb_server_*): minimizations and force + energy
    evaluations.  Submit molecules at any time; completed requests come back from poll() with
    their final coordinates (minimization) or forces (evaluation)."""

    def __init__(self, budget_bytes=2.0e9, max_batch_molecules=512, max_batches=16,
                 cycles_per_launch=50, options: Options | None = None, migrate_fraction=None,
                 **controls):
        lib = library()
        o = ServerOptions()
        lib.sb_default_server_options(ctypes.byref(o))
        if options is not None:
            o.options = options
        for k, v in controls.items():
            setattr(o.controls, k, v)
        o.hbm_budget_bytes = float(budget_bytes)
        o.max_batch_molecules = int(max_batch_molecules)
        o.max_batches = int(max_batches)
        o.cycles_per_launch = int(cycles_per_launch)
        if migrate_fraction is not None:
            o.migrate_fraction = float(migrate_fraction)
        self.options = o
        handle = ctypes.c_void_p()
        _check(lib.sb_server_create(ctypes.byref(o), ctypes.byref(handle)), "sb_server_create")
        self.handle = handle
        self._natom = {}

    def prepare(self, molecule):
        """Topology arrays of a molecule, reusable for many submissions."""
        return _TopologyArrays(molecule)

    def submit(self, molecule, coords=None, prepared=None, evaluate=False):
        """Queue a minimization, or with evaluate=True a force + energy evaluation (its result
        carries the forces where a minimization's carries the final coordinates)."""
        t = prepared if prepared is not None else _TopologyArrays(molecule)
        xyz = np.ascontiguousarray(np.asarray(molecule.coords if coords is None else coords,
                                              dtype=np.float64).reshape(-1))
        rid = ctypes.c_longlong()
        fn = library().sb_server_submit_evaluation if evaluate else library().sb_server_submit
        _check(fn(self.handle, ctypes.byref(t.struct), xyz.ctypes.data, ctypes.byref(rid)),
               "sb_server_submit")
        self._natom[rid.value] = molecule.natom
        return rid.value

    def poll(self, max_results=4096, coordinates=True):
        """List of (result dict, array or None) for the requests completed so far: final
        coordinates of a minimization, forces of an evaluation (dict key "kind").  A request
        that failed has a nonzero "status" (the library's error code) and no array."""
        res = (ServedResult * max_results)()
        cap = 3 * sum(self._natom.values()) if coordinates else 0
        buf = np.zeros(max(cap, 1)) if coordinates else None
        n = ctypes.c_int()
        _check(library().sb_server_poll(self.handle, res, max_results,
                                        buf.ctypes.data if coordinates else None, cap,
                                        ctypes.byref(n)), "sb_server_poll")
        out = []
        off = 0
        for k in range(n.value):
            r = res[k]
            d = {"request_id": r.request_id, "natom": r.natom,
                 "kind": "evaluate" if r.kind == SB_REQUEST_EVALUATE else "minimize",
                 "cycles": r.cycles, "status": r.status,
                 "converged": bool(r.converged), "rms_force": r.rms_force, "energy": r.energy,
                 "energies": np.array(r.energies[:]), "submit_time": r.submit_time,
                 "admit_time": r.admit_time, "finish_time": r.finish_time}
            xyz = None
            if coordinates and r.status == 0:
                xyz = buf[off:off + 3 * r.natom].reshape(-1, 3).copy()
                off += 3 * r.natom
            self._natom.pop(r.request_id, None)
            out.append((d, xyz))
        return out

    def drain(self, timeout=60.0):
        rc = library().sb_server_drain(self.handle, float(timeout))
        if rc == SB_TIMEOUT:
            return False
        _check(rc, "sb_server_drain")
        return True

    def stats(self):
        st = ServerStats()
        _check(library().sb_server_get_stats(self.handle, ctypes.byref(st)), "sb_server_get_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            library().sb_server_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
