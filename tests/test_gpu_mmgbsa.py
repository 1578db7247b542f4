"""The MM-GBSA caller on the GPU: receptor, ligand poses and complexes evaluated (and minimized)
in one synthesis, each system within the per-term bounds of the FP64 oracle."""
import numpy as np
import pytest

import oracle
from stormm_b200 import mmgbsa, synthetic
from fixtures import check_energies, oracle_magnitudes

pytestmark = pytest.mark.gpu


def _poses(r, l, k, rng):
    """Ligand poses beside the receptor: random orientations moved out until no pair is closer
    than 3 A; the last pose far away."""
    out = []
    for p in range(k):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        x = (l.coords - l.coords.mean(0)) @ q.T
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        s = 0.0 if p < k - 1 else 200.0
        while True:
            pose = x + r.coords.mean(0) + d * s
            if np.sqrt(((pose[:, None] - r.coords[None]) ** 2).sum(-1)).min() > 3.0:
                break
            s += 0.5
        out.append(pose)
    return np.array(out)


def test_binding_energies():
    r = synthetic.make_molecule(synthetic._seed(62, 0), 150, noise=0.1)
    l = synthetic.make_molecule(synthetic._seed(62, 1), 32, noise=0.1)
    calc = mmgbsa.MMGBSA(r, l)
    poses = _poses(r, l, 6, np.random.default_rng(3))
    res = calc.run(poses)
    check_energies(res["receptor"], oracle.from_molecule(r).evaluate(r.coords)["energies"],
                   oracle_magnitudes(r), "receptor")
    for p, pose in enumerate(poses):
        ol = oracle.from_molecule(l)
        check_energies(res["ligand"][p], ol.evaluate(pose)["energies"],
                       ol.magnitudes(pose), f"ligand {p}")
        c = mmgbsa.combine(r, l, pose)
        oc = oracle.from_molecule(c)
        check_energies(res["complex"][p], oc.evaluate(c.coords)["energies"],
                       oc.magnitudes(c.coords), f"complex {p}")
    np.testing.assert_allclose(res["binding"], res["binding_terms"].sum(axis=1))
    assert abs(res["binding"][-1]) < 5e-3           # the far pose barely interacts
    assert np.abs(res["binding"][:-1]).max() > 0.5   # contact poses do
    # minimized: every system's energy drops
    res_min = calc.run(poses, minimize_cycles=40, sd_cycles=10)
    assert (res_min["complex"].sum(axis=1) < res["complex"].sum(axis=1)).all()
    assert res_min["receptor"].sum() < res["receptor"].sum()


def test_surface_area_term():
    """With sphere points (STORMM's 272-point set from the surface-area fixture) every system's
    surface-area energy equals the oracle's restatement of STORMM's surfaceArea at the same
    coordinates, and the binding energy takes the complex's minus the parts'."""
    from fixtures import load
    pts = load("sasa_s60.npz")["sphere_points"]
    r = synthetic.make_molecule(synthetic._seed(62, 0), 150, noise=0.1)
    l = synthetic.make_molecule(synthetic._seed(62, 1), 32, noise=0.1)
    calc = mmgbsa.MMGBSA(r, l)
    poses = _poses(r, l, 3, np.random.default_rng(4))
    plain = calc.run(poses)
    res = calc.run(poses, sphere_points=pts)
    # the oracle takes the synthesis's own (fixed-point) coordinates
    parts = [r] + [l] * len(poses) + [calc.complex] * len(poses)
    for k, m in enumerate(parts):
        x = np.asarray(res["coordinates"][k]).reshape(-1, 3)
        want = oracle.surface_area(x, oracle.sasa_radii(m), pts, weight=0.005)
        assert abs(res["surface_area"][k] - want) <= 1e-10 * want, k
    k = len(poses)
    sa = res["surface_area"]
    np.testing.assert_allclose(res["binding"] - plain["binding"],
                               sa[1 + k:] - sa[0] - sa[1:1 + k], rtol=0, atol=1e-12)
