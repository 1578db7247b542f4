"""The conformer-search caller (stormm_b200.conformers) on the host: its clash test and RMSD
against STORMM's own (fixture from tests/golden/make_conformer_golden.py), the geometry of its
replicas, and its selection rule.  The batched minimization between them runs in
tests/test_gpu_conformers.py."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from stormm_b200 import conformers as cf
from stormm_b200 import synthetic


def _fixture():
    return dict(np.load(os.path.join(GOLDEN, "conformer_geometry.npz")))


@pytest.mark.parametrize("case", [0, 1], ids=["48 atoms (grid path)", "24 atoms (direct path)"])
def test_clash_and_rmsd_match_stormm(case):
    """detectClash verdicts and ALIGN_MASS RMSDs of STORMM's CPU build on 71 geometries per
    molecule, clashing and not: the verdicts equal, the RMSDs to 1e-12 A."""
    g = _fixture()
    m = synthetic.make_molecule(synthetic._seed(int(g[f"seed{case}"]), 0), int(g[f"natom{case}"]),
                                noise=0.1)
    lim = cf._clash_limits(m)
    coords = g[f"coords{case}"]
    ours = np.array([cf.clashes(c, lim) for c in coords])
    np.testing.assert_array_equal(ours, g[f"clash{case}"].astype(bool))
    assert 0 < ours.sum() < len(ours)
    rmsd = np.array([cf.aligned_rmsd(coords[0], c, m.mass) for c in coords])
    np.testing.assert_allclose(rmsd, g[f"rmsd{case}"], rtol=0, atol=1e-12)


def test_rotatable_bonds_and_turns():
    """Ring and terminal bonds are not rotatable; a turn moves the smaller side rigidly and keeps
    the bond lengths."""
    # a chain 0-1-2-3-4 with a ring 4-5-6-7-4 and a hydrogen-like end 8 on 0
    bonds = np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 5], [5, 6], [6, 7], [7, 4], [0, 8]])
    rb = cf.rotatable_bonds(9, bonds)
    pairs = {tuple(sorted((i, j))) for i, j, _ in rb}
    assert pairs == {(0, 1), (1, 2), (2, 3), (3, 4)}
    for i, j, moved in rb:
        assert len(moved) <= 9 - len(moved) and j in moved and i not in moved
    rng = np.random.default_rng(0)
    xyz = rng.normal(size=(9, 3)) * 2.0
    i, j, moved = rb[0]
    out = cf.rotate_about_bond(xyz, i, j, moved, 2.0)
    fixed = np.setdiff1d(np.arange(9), moved)
    np.testing.assert_allclose(out[fixed], xyz[fixed])
    dist = lambda c, a, b: np.linalg.norm(c[a] - c[b])
    for a, b in bonds:
        assert dist(out, a, b) == pytest.approx(dist(xyz, a, b), abs=1e-12)
    assert not np.allclose(out[moved], xyz[moved])


def test_replicas_are_clash_free_and_varied():
    m = synthetic.make_molecule(synthetic._seed(32, 0), 64, noise=0.1)
    s = cf.ConformerSearch(m, replicas=32, seed=3)
    assert not any(cf.clashes(x, s.limits) for x in s.start)
    rmsd = [cf.aligned_rmsd(m.coords, x, m.mass) for x in s.start]
    assert np.median(rmsd) > 0.5


def test_selection_rule():
    """filterMinimizedStructures: lowest energy first, nothing that clashes, nothing within the
    RMSD tolerance of a structure kept before it, and every structure left out either clashes or
    lies within the tolerance of a kept one of no higher energy (or the count was reached)."""
    rng = np.random.default_rng(4)
    m = synthetic.make_molecule(synthetic._seed(33, 0), 30, noise=0.1)
    coords = np.array([m.coords + rng.normal(scale=rng.uniform(0.05, 1.5), size=m.coords.shape)
                       for _ in range(40)])
    energies = rng.normal(size=40)
    clashing = rng.random(40) < 0.2
    tol = 0.9
    kept = cf.select_conformers(energies, coords, m.mass, clashing, 100, tol)
    assert kept and not clashing[kept].any()
    assert list(np.argsort(energies[kept], kind="stable")) == list(range(len(kept)))
    for a in range(len(kept)):
        for b in range(a + 1, len(kept)):
            assert cf.aligned_rmsd(coords[kept[a]], coords[kept[b]], m.mass) >= tol
    for k in set(range(40)) - set(kept):
        if clashing[k]:
            continue
        assert any(cf.aligned_rmsd(coords[s], coords[k], m.mass) < tol and energies[s] <= energies[k]
                   for s in kept)
    assert cf.select_conformers(energies, coords, m.mass, clashing, 3, tol) == kept[:3]
