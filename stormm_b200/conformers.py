"""Conformer search on the batched minimizer: the caller STORMM's conformer application is
(apps/Conf/src/conformer.cpp:118-215), on this library.

  search = ConformerSearch(molecule, replicas=512, seed=1)
  result = search.run(final_states=20)        # ConformerResult: energies, coordinates, ...

The steps follow the application's:

1. Sampling workspace (apps/Conf/src/setup.cpp:126-160, buildSamplingWorkspace): replicas of
   the molecule, each with its rotatable bonds turned in turn by seeded choices among
   rotation_samples evenly spaced angles; a turn that makes the geometry clash is drawn again
   (at most max_attempts times, after which that bond keeps its setting).  Rotatable bonds: acyclic
   bonds between two atoms that each have another neighbour; at most max_rotatable_bonds of
   them, those that move the most atoms' smaller side first; a turn moves the smaller side.
2. One synthesis of all replicas (one shared topology) minimized in one batched run
   (launchMinimization in the application; Synthesis.minimize here).
3. Selection (apps/Conf/src/analysis.cpp:75-237, filterMinimizedStructures): structures that
   clash after minimization (detectClash, Structure/clash_detection.h; see _clash_limits for
   the criterion it applies) are dropped; then, final_states times, the lowest-energy remaining structure is kept and
   every structure within rmsd_tolerance of it (mass-weighted positional RMSD after optimal
   superposition, RMSDMethod::ALIGN_MASS) is eliminated.

The replica generator is this module's own: STORMM's draws its rotation settings through its
SynthesisPermutor with cis-trans and chirality options that the synthetic molecules here never
need.  The minimizer and the selection are the application's.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# apps/Conf defaults (Namelists/nml_conformer.h:26-47) and the clash criterion's defaults
# (default_minimize_clash_r0 / default_minimize_clash_ratio, Namelists/nml_minimize.h)
DEFAULT_ROTATION_SAMPLES = 3
DEFAULT_MAX_ROTATABLE_BONDS = 4
DEFAULT_FINAL_STATES = 100
DEFAULT_RMSD_TOLERANCE = 1.5
CLASH_DISTANCE = 0.2
CLASH_RATIO = 0.5


def rotatable_bonds(natom, bonds):
    """Acyclic bonds (i, j) between atoms that each have another neighbour, with the atoms on
    j's side of the bond (the side a turn moves, the smaller one)."""
    nbr = [[] for _ in range(natom)]
    for i, j in bonds:
        nbr[int(i)].append(int(j))
        nbr[int(j)].append(int(i))
    out = []
    for i, j in bonds:
        i, j = int(i), int(j)
        if len(nbr[i]) < 2 or len(nbr[j]) < 2:
            continue
        # atoms reachable from j without crossing the bond
        side, stack = {j}, [j]
        cyclic = False
        while stack and not cyclic:
            a = stack.pop()
            for b in nbr[a]:
                if a == j and b == i:
                    continue
                if b == i:
                    cyclic = True        # j reaches i another way: the bond is in a ring
                    break
                if b not in side:
                    side.add(b)
                    stack.append(b)
        if cyclic:
            continue
        if len(side) > natom - len(side):
            side = set(range(natom)) - side
            i, j = j, i
        out.append((i, j, np.array(sorted(side), dtype=np.int64)))
    # the bonds that move the most atoms first
    out.sort(key=lambda t: (-len(t[2]), t[0], t[1]))
    return out


def rotate_about_bond(xyz, i, j, moved, angle):
    """Coordinates with the atoms `moved` turned by `angle` radians about the axis i -> j."""
    out = np.array(xyz, dtype=np.float64, copy=True)
    axis = out[j] - out[i]
    axis /= np.linalg.norm(axis)
    c, s = np.cos(angle), np.sin(angle)
    p = out[moved] - out[j]
    # Rodrigues' rotation formula
    out[moved] = (out[j] + p * c + np.cross(axis, p) * s +
                  np.outer(p @ axis, axis) * (1.0 - c))
    return out


def _excluded(mol):
    ex = [set(mol.excl12[a]) | set(mol.excl13[a]) | set(mol.excl14[a]) for a in range(mol.natom)]
    return ex


def _sigma(a, b):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(b > 0.0, (a / np.where(b > 0.0, b, 1.0)) ** (1.0 / 6.0), 0.0)


def _clash_limits(mol):
    """Per pair, the distance below which it clashes, as STORMM's detectClash decides
    (Structure/clash_detection.tpp:66-175, 251-300, 316-441): the 1-4 pairs of dihedrals below
    the clash ratio times their 1-4 sigma = (A14 / B14)^(1/6); other excluded pairs never; the
    remaining pairs below the larger of a distance and a ratio times their sigma.  For those
    detectClash hands its clash distance and ratio to the pair tests in swapped order
    (clash_detection.tpp:329-330, 362-395: the tests take (elec_limit, vdw_ratio), the calls
    pass (vdw_ratio, elec_limit)), so with the defaults a pair clashes below 0.5 A or 0.2
    sigma; the limits here reproduce that, so that the structures dropped are the
    application's."""
    n = mol.natom
    t = mol.lj_idx
    lim = np.maximum(CLASH_RATIO,
                     CLASH_DISTANCE * _sigma(mol.lja[t[:, None], t[None, :]],
                                             mol.ljb[t[:, None], t[None, :]]))
    for i, ex in enumerate(_excluded(mol)):
        for j in ex:
            lim[i, j] = 0.0
    lim[np.arange(n), np.arange(n)] = 0.0
    a14 = getattr(mol, "lja14", None)
    b14 = getattr(mol, "ljb14", None)
    a14 = mol.lja if a14 is None else a14
    b14 = mol.ljb if b14 is None else b14
    for d, has14 in zip(mol.dihedrals, mol.dihe_has14):
        if has14:
            i, l = int(d[0]), int(d[3])
            lim[i, l] = lim[l, i] = CLASH_RATIO * float(_sigma(a14[t[i], t[l]], b14[t[i], t[l]]))
    return lim


def clashes(xyz, limits):
    """True when a pair of atoms sits closer than its clash limit (detectClash)."""
    d = np.sqrt(((xyz[:, None, :] - xyz[None, :, :]) ** 2).sum(-1))
    return bool((d < limits).any())


def aligned_rmsd(a, b, masses):
    """Mass-weighted positional RMSD of b against a after optimal superposition (Kabsch)."""
    w = masses / masses.sum()
    ca = (a * w[:, None]).sum(0)
    cb = (b * w[:, None]).sum(0)
    pa, pb = a - ca, b - cb
    h = (pb * w[:, None]).T @ pa
    u, _, vt = np.linalg.svd(h)
    d = np.sign(np.linalg.det(vt.T @ u.T))
    r = vt.T @ np.diag([1.0, 1.0, d]) @ u.T
    diff = pb @ r.T - pa
    return float(np.sqrt((w * (diff ** 2).sum(1)).sum()))


def select_conformers(energies, coords, masses, clashing, final_states, rmsd_tolerance):
    """Indices of the conformers kept, in the order found (filterMinimizedStructures): the
    lowest-energy structure that neither clashes nor lies within rmsd_tolerance of one already
    kept, repeated up to final_states times.  Ties go to the lower index."""
    n = len(energies)
    alive = ~np.asarray(clashing, dtype=bool)
    kept = []
    for _ in range(final_states):
        cand = np.flatnonzero(alive)
        if cand.size == 0:
            break
        best = int(cand[np.argmin(np.asarray(energies)[cand])])
        kept.append(best)
        for k in cand:
            if aligned_rmsd(coords[best], coords[k], masses) < rmsd_tolerance:
                alive[k] = False
        alive[best] = False
    assert len(kept) <= n
    return kept


@dataclass
class ConformerResult:
    selected: list            # indices of the kept replicas, lowest energy first
    energies: np.ndarray      # final total energy of every replica (kcal/mol)
    coordinates: np.ndarray   # (replicas, natom, 3) final coordinates
    clashing: np.ndarray      # replicas dropped for clashes after minimization
    start: np.ndarray         # (replicas, natom, 3) starting coordinates
    history: np.ndarray | None


class ConformerSearch:
    """Replicas of one molecule turned about its rotatable bonds, minimized together on the GPU,
    then filtered by energy and RMSD as STORMM's conformer application does."""

    def __init__(self, molecule, replicas=512, seed=1,
                 rotation_samples=DEFAULT_ROTATION_SAMPLES,
                 max_rotatable_bonds=DEFAULT_MAX_ROTATABLE_BONDS, max_attempts=3):
        self.mol = molecule
        self.replicas = int(replicas)
        self.limits = _clash_limits(molecule)
        self.bonds = rotatable_bonds(molecule.natom, molecule.bonds)[:max_rotatable_bonds]
        rng = np.random.default_rng(seed)
        angles = 2.0 * np.pi * np.arange(rotation_samples) / rotation_samples
        start = np.empty((self.replicas, molecule.natom, 3))
        for r in range(self.replicas):
            xyz = np.array(molecule.coords, dtype=np.float64, copy=True)
            for (i, j, moved) in self.bonds:
                for _ in range(max_attempts):
                    trial = rotate_about_bond(xyz, i, j, moved,
                                              angles[rng.integers(rotation_samples)])
                    if not clashes(trial, self.limits):
                        xyz = trial
                        break
            start[r] = xyz
        self.start = start

    def run(self, final_states=DEFAULT_FINAL_STATES, rmsd_tolerance=DEFAULT_RMSD_TOLERANCE,
            options=None, record_history=False, **controls):
        """Minimize every replica in one batch (STORMM's minimizer defaults, overridable by
        MinimizeControls field names) and select the conformers."""
        import stormm_b200 as sb
        syn = sb.Synthesis([self.mol], topology_index=np.zeros(self.replicas, dtype=np.int32),
                           options=options)
        try:
            syn.set_coordinates(self.start)
            syn.minimize(record_history=record_history, **controls)
            history = syn.minimize_history() if record_history else None
            coords = syn.coordinates().reshape(self.replicas, self.mol.natom, 3)
            energies = syn.energy_terms().sum(axis=1)
        finally:
            syn.close()
        clashing = np.array([clashes(c, self.limits) for c in coords])
        selected = select_conformers(energies, coords, self.mol.mass, clashing, final_states,
                                     rmsd_tolerance)
        return ConformerResult(selected, energies, coords, clashing, self.start, history)
