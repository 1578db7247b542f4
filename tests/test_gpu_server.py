"""The request server (continuous batching of minimization requests) on the GPU.

Each served molecule must come back exactly as it does when minimized alone: trajectories are
per molecule, every sum is order-independent and the minimizer state persists between launches,
so the coordinates, cycle counts and energies are bit-identical whatever batch, backfill or
launch split a request gets."""
import time

import numpy as np
import pytest

import stormm_b200 as sb
from stormm_b200 import synthetic

pytestmark = pytest.mark.gpu

CONTROLS = dict(total_cycles=150, sd_cycles=30, convergence_rms=0.5, kernel=sb.MIN_PERSISTENT)


def _alone(mol):
    syn = sb.Synthesis([mol])
    syn.set_coordinates(mol.coords)
    syn.minimize(**CONTROLS)
    cycles, conv, _ = syn.minimize_progress()
    out = (syn.coordinates().copy(), syn.energies()[0].copy(), int(cycles[0]), bool(conv[0]))
    syn.close()
    return out


def test_served_results_equal_alone_results():
    sizes = [12, 30, 48, 64, 33, 96, 140, 257, 20, 75]
    mols = [synthetic.make_molecule(synthetic._seed(8080, k), n, 0.3)
            for k, n in enumerate(sizes)]
    srv = sb.Server(max_batch_molecules=3, max_batches=4, cycles_per_launch=20, **CONTROLS)
    ids = {}
    for m in mols[:5]:
        ids[srv.submit(m)] = m
    time.sleep(0.05)                 # the first batches are running when the rest arrive
    for m in mols[5:]:
        ids[srv.submit(m)] = m
    assert srv.drain(120.0)
    results = srv.poll()
    assert len(results) == len(mols)
    st = srv.stats()
    assert st["completed"] == len(mols) and st["in_flight"] == 0 and st["pending"] == 0
    srv.close()
    for r, xyz in results:
        m = ids[r["request_id"]]
        c_alone, e_alone, cyc_alone, conv_alone = _alone(m)
        assert r["natom"] == m.natom
        assert r["cycles"] == cyc_alone and r["converged"] == conv_alone
        assert np.array_equal(xyz, c_alone)
        assert np.array_equal(r["energies"], e_alone)
        assert r["energy"] == pytest.approx(e_alone.sum(), rel=1e-12, abs=1e-9)
        assert r["submit_time"] <= r["admit_time"] <= r["finish_time"]


def test_budget_bounds_the_molecules_in_flight():
    mols = [synthetic.make_molecule(synthetic._seed(9090, k), 40, 0.3) for k in range(8)]
    probe = sb.Server(budget_bytes=1.0e9, **CONTROLS)
    probe.close()
    # room for two 40-atom molecules at a time (about 48 KB each)
    srv = sb.Server(budget_bytes=100000.0, max_batch_molecules=8, cycles_per_launch=10,
                    **CONTROLS)
    for m in mols:
        srv.submit(m)
    peak = 0.0
    t_end = time.time() + 120.0
    while time.time() < t_end:
        st = srv.stats()
        peak = max(peak, st["bytes_in_flight"])
        if st["completed"] == len(mols):
            break
        time.sleep(0.002)
    assert srv.drain(60.0)
    assert len(srv.poll()) == len(mols)
    assert 0.0 < peak <= 100000.0
    big = synthetic.make_molecule(1, 300, 0.1)
    with pytest.raises(sb.StormmB200Error):
        srv.submit(big)
    srv.close()
