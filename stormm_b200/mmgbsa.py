"""MM-GBSA binding energies on the batched path: the caller STORMM's MM-GBSA application is
(apps/Gbsa/src/mmgbsa.cpp:180-275), on this library.

  calc = MMGBSA(receptor, ligand)                 # molecule objects (topology + coordinates)
  res = calc.run(poses)                           # poses: (k, ligand atoms, 3) in the receptor
  res["binding"]                                  # per pose: E_complex - E_receptor - E_ligand

As in the application, one synthesis holds the receptor, every ligand pose and every complex
(receptor first, then the pose's ligand: the order of STORMM's combined AtomGraph), so the three
kinds of system are evaluated, or minimized (minimize_cycles > 0) and then evaluated, together;
the binding energy of a pose is the complex's energy minus those of the receptor and the ligand,
term by term.  The complex's topology joins the two molecules: their atoms, valence terms and
exclusions side by side, and a Lennard-Jones table over both molecules' types whose blocks for
each molecule are that molecule's own table and whose cross blocks follow the Lorentz-Berthelot
rules from each type's sigma and epsilon (the rules of the force fields here; STORMM's
combination of topologies infers the rule from the tables, Topology/combograph_ljmodel.cpp).
The surface-area term (apps/Gbsa/src/mmgbsa.cpp:244-253: surfaceArea over every molecule,
probe 1.4 A, 0.005 kcal/mol per A^2) is added when the caller passes the sphere points
(sphere_points, unit vectors; STORMM's application places 272 by its geodesic polyhedron),
computed on the GPU for every system of the batch at the final coordinates.
Not computed here: the application's carve-out of the binding site.
"""
from __future__ import annotations

import numpy as np

from stormm_b200 import synthetic


def _type_parameters(a, b):
    """Per type sigma and epsilon from the diagonal of an (A, B) table (A = 4 eps sigma^12,
    B = 4 eps sigma^6); zero for a type without Lennard-Jones."""
    da, db = np.diag(a), np.diag(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        sigma = np.where(db > 0.0, (da / np.where(db > 0.0, db, 1.0)) ** (1.0 / 6.0), 0.0)
        eps = np.where(da > 0.0, db * db / (4.0 * np.where(da > 0.0, da, 1.0)), 0.0)
    return sigma, eps


def _joined_table(a1, b1, a2, b2):
    n1, n2 = a1.shape[0], a2.shape[0]
    s1, e1 = _type_parameters(a1, b1)
    s2, e2 = _type_parameters(a2, b2)
    sig = 0.5 * (s1[:, None] + s2[None, :])
    eps = np.sqrt(e1[:, None] * e2[None, :])
    ca = 4.0 * eps * sig ** 12
    cb = 4.0 * eps * sig ** 6
    a = np.zeros((n1 + n2, n1 + n2))
    b = np.zeros((n1 + n2, n1 + n2))
    a[:n1, :n1], b[:n1, :n1] = a1, b1
    a[n1:, n1:], b[n1:, n1:] = a2, b2
    a[:n1, n1:], b[:n1, n1:] = ca, cb
    a[n1:, :n1], b[n1:, :n1] = ca.T, cb.T
    return a, b


def combine(receptor, ligand, ligand_coords=None, name="complex"):
    """The complex of the two molecules: receptor atoms first, then the ligand's."""
    r, l = receptor, ligand
    n = r.natom
    lc = l.coords if ligand_coords is None else np.asarray(ligand_coords, dtype=np.float64)
    lja, ljb = _joined_table(r.lja, r.ljb, l.lja, l.ljb)
    fields = dict(
        natom=r.natom + l.natom,
        coords=np.concatenate([r.coords, lc]),
        charge=np.concatenate([r.charge, l.charge]),
        lj_idx=np.concatenate([r.lj_idx, l.lj_idx + r.n_lj_types]).astype(np.int32),
        lja=lja, ljb=ljb,
        z_numbers=np.concatenate([r.z_numbers, l.z_numbers]).astype(np.int32),
        mass=np.concatenate([r.mass, l.mass]),
        pb_radii=np.concatenate([r.pb_radii, l.pb_radii]),
        gb_screen=np.concatenate([r.gb_screen, l.gb_screen]),
        bonds=np.concatenate([r.bonds, l.bonds + n]).astype(np.int32),
        bond_k=np.concatenate([r.bond_k, l.bond_k]),
        bond_r0=np.concatenate([r.bond_r0, l.bond_r0]),
        angles=np.concatenate([r.angles, l.angles + n]).astype(np.int32),
        angl_k=np.concatenate([r.angl_k, l.angl_k]),
        angl_theta0=np.concatenate([r.angl_theta0, l.angl_theta0]),
        dihedrals=np.concatenate([r.dihedrals, l.dihedrals + n]).astype(np.int32),
        dihe_amp=np.concatenate([r.dihe_amp, l.dihe_amp]),
        dihe_freq=np.concatenate([r.dihe_freq, l.dihe_freq]),
        dihe_phase=np.concatenate([r.dihe_phase, l.dihe_phase]),
        dihe_has14=np.concatenate([r.dihe_has14, l.dihe_has14]),
        scee=r.scee, scnb=r.scnb, name=name)
    if r.scee != l.scee or r.scnb != l.scnb:
        raise ValueError("receptor and ligand must share their 1-4 scaling factors")
    for extra in ("dihe_improper", "gb_alpha", "gb_beta", "gb_gamma"):
        rv, lv = getattr(r, extra, None), getattr(l, extra, None)
        if (rv is None) != (lv is None):
            raise ValueError(f"{extra} present in one molecule only")
    e12, e13, e14 = synthetic.exclusion_lists(fields["natom"], fields["bonds"])
    m = synthetic.Molecule(**fields, excl12=e12, excl13=e13, excl14=e14)
    for extra in ("dihe_improper", "gb_alpha", "gb_beta", "gb_gamma"):
        rv, lv = getattr(r, extra, None), getattr(l, extra, None)
        if rv is not None:
            setattr(m, extra, np.concatenate([rv, lv]))
    return m


class MMGBSA:
    """Receptor, ligand poses and complexes in one synthesis (one topology each for the
    receptor, the ligand and the complex)."""

    def __init__(self, receptor, ligand):
        self.receptor = receptor
        self.ligand = ligand
        self.complex = combine(receptor, ligand)

    def run(self, poses, minimize_cycles=0, options=None, sphere_points=None,
            probe_radius=1.4, sasa_weight=0.005, **controls):
        """Energies of the receptor, each ligand pose and each complex (after minimize_cycles
        line-minimization cycles when positive), and the binding energy of each pose; with
        sphere_points, the surface-area energy of each system joins them."""
        import stormm_b200 as sb
        poses = np.asarray(poses, dtype=np.float64).reshape(-1, self.ligand.natom, 3)
        k = len(poses)
        index = np.concatenate([[0], np.ones(k, dtype=np.int32), np.full(k, 2, dtype=np.int32)])
        syn = sb.Synthesis([self.receptor, self.ligand, self.complex], topology_index=index,
                           options=options)
        try:
            xyz = np.concatenate([self.receptor.coords.reshape(-1, 3)] + list(poses) +
                                 [np.concatenate([self.receptor.coords, p]) for p in poses])
            syn.set_coordinates(xyz)
            if minimize_cycles > 0:
                syn.minimize(total_cycles=minimize_cycles, **controls)
            syn.initialize()
            syn.evaluate()
            e = syn.energy_terms()
            coords = syn.split(syn.coordinates())
            sa = None
            if sphere_points is not None:
                sa = syn.surface_area(sphere_points, probe_radius, sasa_weight)
        finally:
            syn.close()
        rec, lig, cpx = e[0], e[1:1 + k], e[1 + k:]
        binding_terms = cpx - rec[None, :] - lig
        out = {"receptor": rec, "ligand": lig, "complex": cpx,
               "binding_terms": binding_terms, "binding": binding_terms.sum(axis=1),
               "coordinates": coords}
        if sa is not None:
            out["surface_area"] = sa
            out["binding_surface_area"] = sa[1 + k:] - sa[0] - sa[1:1 + k]
            out["binding"] = out["binding"] + out["binding_surface_area"]
        return out
