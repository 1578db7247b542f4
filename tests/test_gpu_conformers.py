"""The conformer-search caller on the GPU: replicas of one molecule minimized in one batch (one
shared topology), then selected as STORMM's conformer application selects them."""
import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from stormm_b200 import conformers as cf
from stormm_b200 import synthetic
from fixtures import check_energies, oracle_magnitudes

pytestmark = pytest.mark.gpu

CONTROLS = dict(total_cycles=120, sd_cycles=30)


def test_conformer_search_minimizes_and_selects():
    m = synthetic.make_molecule(synthetic._seed(91, 0), 44, noise=0.1)
    search = cf.ConformerSearch(m, replicas=48, seed=5)
    res = search.run(final_states=8, rmsd_tolerance=0.75, **CONTROLS)
    osys = oracle.from_molecule(m)
    e0 = np.array([osys.evaluate(x, forces=False)["energies"].sum() for x in search.start])
    # the minimizer lowers every replica's energy
    assert (res.energies < e0).all()
    # each replica's reported energy is that of its final coordinates (FP64 oracle, per-term
    # bounds of the single-point tests)
    for k in (0, 17, 31):
        o = osys.evaluate(res.coordinates[k])
        syn = sb.Synthesis([m])
        syn.set_coordinates(res.coordinates[k])
        syn.initialize()
        syn.evaluate()
        check_energies(syn.energy_terms()[0], o["energies"],
                       oracle_magnitudes(m, res.coordinates[k]), f"replica {k}")
        syn.close()
    # a replica minimized alone ends bit for bit where the batch put it
    one = sb.Synthesis([m])
    one.set_coordinates(search.start[17])
    one.minimize(**CONTROLS)
    np.testing.assert_array_equal(one.coordinates().reshape(-1, 3), res.coordinates[17])
    one.close()
    # the selection: lowest energies first, no clash, separated by the RMSD tolerance
    kept = res.selected
    assert 0 < len(kept) <= 8 and not res.clashing[kept].any()
    assert kept[0] == int(np.argmin(np.where(res.clashing, np.inf, res.energies)))
    assert list(np.diff(res.energies[kept]) >= 0) == [True] * (len(kept) - 1)
    for a in range(len(kept)):
        for b in range(a + 1, len(kept)):
            assert cf.aligned_rmsd(res.coordinates[kept[a]], res.coordinates[kept[b]],
                                   m.mass) >= 0.75
