"""The MM-GBSA caller's complex topology (stormm_b200.mmgbsa.combine) on the host, against the
FP64 oracle: the complex carries both molecules' terms unchanged, and a ligand far from the
receptor leaves only the vanishing cross terms.  tests/test_gpu_mmgbsa.py runs the batched
evaluation."""
import numpy as np

import oracle
from stormm_b200 import mmgbsa, synthetic


def _pair():
    r = synthetic.make_molecule(synthetic._seed(61, 0), 120, noise=0.1)
    l = synthetic.make_molecule(synthetic._seed(61, 1), 30, noise=0.1)
    return r, l


def test_lennard_jones_blocks():
    """The molecules' own tables sit on the diagonal blocks; the cross blocks follow the
    Lorentz-Berthelot rules, which also reproduce each molecule's own off-diagonal entries."""
    r, l = _pair()
    c = mmgbsa.combine(r, l)
    nr = r.n_lj_types
    np.testing.assert_array_equal(c.lja[:nr, :nr], r.lja)
    np.testing.assert_array_equal(c.ljb[nr:, nr:], l.ljb)
    own = mmgbsa._joined_table(r.lja, r.ljb, r.lja, r.ljb)
    np.testing.assert_allclose(own[0][:nr, nr:], r.lja, rtol=1e-7)
    np.testing.assert_allclose(own[1][:nr, nr:], r.ljb, rtol=1e-7)


def test_complex_terms_and_far_ligand():
    r, l = _pair()
    far = l.coords + np.array([250.0, 0.0, 0.0])
    c = mmgbsa.combine(r, l, far)
    ec = oracle.from_molecule(c).evaluate(c.coords)["energies"]
    er = oracle.from_molecule(r).evaluate(r.coords)["energies"]
    el = oracle.from_molecule(l).evaluate(far)["energies"]
    # bonds, angles, dihedrals and 1-4 terms: the sums of the parts
    for t in (0, 1, 2, 3, 5, 7):
        assert abs(ec[t] - er[t] - el[t]) <= 1e-9 * max(1.0, abs(ec[t]))
    # nonbonded and GB cross terms vanish with distance (neutral molecules)
    assert np.abs(ec - er - el).max() < 2e-3
