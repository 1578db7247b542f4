"""The request server (continuous batching of minimization requests) on the GPU.

Each served molecule must come back exactly as it does when minimized alone: trajectories are
per molecule, every sum is order-independent and the minimizer state persists between launches,
so the coordinates, cycle counts and energies are bit-identical whatever batch, backfill or
launch split a request gets."""
import copy
import time

import numpy as np
import pytest

import stormm_b200 as sb
from stormm_b200 import synthetic
from fixtures import check_energies, oracle_magnitudes

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


def _evaluated_alone(mol):
    syn = sb.Synthesis([mol])
    syn.set_coordinates(mol.coords)
    syn.initialize()
    syn.evaluate()
    out = (syn.forces().copy(), syn.energies()[0].copy())
    syn.close()
    return out


def test_evaluation_requests_mixed_with_minimizations():
    """Force + energy requests share the server with minimizations: they batch with each other,
    overlap with the minimization batches in flight, and each comes back exactly as a direct
    evaluation of the molecule alone (and within the oracle's tolerance), as does each
    minimization."""
    import oracle
    sizes = [16, 40, 64, 100, 23, 180, 2600, 48]      # 2,600 atoms goes to the tiled path
    mols = [synthetic.make_molecule(synthetic._seed(7070, k), n, 0.3)
            for k, n in enumerate(sizes[:-2])]
    mols.append(synthetic.make_chain(synthetic._seed(7070, 6), sizes[6]))
    mols.append(synthetic.make_molecule(synthetic._seed(7070, 7), sizes[7], 0.3))
    srv = sb.Server(max_batch_molecules=3, max_batches=4, cycles_per_launch=20, **CONTROLS)
    kinds = {}
    for k, m in enumerate(mols):
        if m.natom <= 2048:
            kinds[srv.submit(m)] = ("minimize", m)
        kinds[srv.submit(m, evaluate=True)] = ("evaluate", m)
        if k == 3:
            time.sleep(0.05)
    assert srv.drain(120.0)
    results = srv.poll()
    srv.close()
    assert len(results) == len(kinds)
    seen = {"minimize": 0, "evaluate": 0}
    for r, arr in results:
        kind, m = kinds[r["request_id"]]
        assert r["kind"] == kind
        seen[kind] += 1
        if kind == "minimize":
            c_alone, e_alone, cyc_alone, _ = _alone(m)
            assert np.array_equal(arr, c_alone) and np.array_equal(r["energies"], e_alone)
            assert r["cycles"] == cyc_alone
            continue
        f_alone, e_alone = _evaluated_alone(m)
        assert np.array_equal(arr, f_alone)
        assert np.array_equal(r["energies"], e_alone)
        assert r["cycles"] == 0
        assert r["rms_force"] == pytest.approx(np.sqrt((f_alone ** 2).mean()), rel=1e-12)
        o = oracle.from_molecule(m).evaluate(m.coords)
        got = np.array([r["energies"][sb.NRG_SLOTS[t]] for t in sb.TERM_ORDER])
        check_energies(got, o["energies"], oracle_magnitudes(m), m.natom)
        err = np.sqrt(((arr - o["forces"]) ** 2).sum() / (o["forces"] ** 2).sum())
        assert err <= 5e-6, (m.natom, err)
    assert seen == {"minimize": len(mols) - 1, "evaluate": len(mols)}


def test_minimization_of_a_large_molecule_is_refused_at_submit():
    big = synthetic.make_chain(synthetic._seed(7171, 0), 2600)
    srv = sb.Server(**CONTROLS)
    with pytest.raises(sb.StormmB200Error, match="cannot be minimized by the persistent"):
        srv.submit(big)
    rid = srv.submit(big, evaluate=True)          # an evaluation of it is served
    assert srv.drain(60.0)
    (r, f), = srv.poll()
    assert r["request_id"] == rid and f.shape == (2600, 3)
    srv.close()


def test_graph_kernel_server_minimizes_a_large_molecule():
    big = synthetic.make_chain(synthetic._seed(7171, 1), 2300, 0.2)
    small = synthetic.make_molecule(synthetic._seed(7171, 2), 60, 0.3)
    controls = dict(total_cycles=30, sd_cycles=10, convergence_rms=0.0, kernel=sb.MIN_GRAPH)
    srv = sb.Server(cycles_per_launch=10, **controls)
    ids = {srv.submit(big): big, srv.submit(small): small}
    assert srv.drain(120.0)
    results = srv.poll()
    srv.close()
    assert len(results) == 2
    for r, xyz in results:
        m = ids[r["request_id"]]
        alone = sb.Synthesis([m])
        alone.set_coordinates(m.coords)
        alone.minimize(**controls)
        assert r["cycles"] == 30
        assert np.array_equal(xyz, alone.coordinates())
        assert np.array_equal(r["energies"], alone.energies()[0])


def _widened_lj(mol, ntypes):
    """The molecule with its Lennard-Jones tables padded to ntypes types (atoms keep theirs)."""
    m = copy.deepcopy(mol)
    nt = mol.lja.shape[0]
    for name in ("lja", "ljb"):
        t = np.full((ntypes, ntypes), 1.0)
        t[:nt, :nt] = getattr(mol, name)
        setattr(m, name, t)
    return m


def test_bad_requests_fail_alone():
    """A malformed topology is refused at submit.  A molecule that passes the host checks but
    cannot be built (its Lennard-Jones tables and atoms need more shared memory than a block
    has) fails with its error code in the result, alone: the batch it was admitted with is
    retried one request per batch, and every good request queued around it comes back exactly
    as it does alone."""
    good = [synthetic.make_molecule(synthetic._seed(6060, k), n, 0.3)
            for k, n in enumerate([20, 44, 70, 33, 90])]
    bad_type = copy.deepcopy(good[0])
    bad_type.lj_idx = bad_type.lj_idx.copy()
    bad_type.lj_idx[3] = bad_type.n_lj_types + 2
    bad_excl = copy.deepcopy(good[1])
    bad_excl.excl12 = [list(e) for e in bad_excl.excl12]
    bad_excl.excl12[0].append(bad_excl.natom + 7)
    unbuildable = _widened_lj(synthetic.make_molecule(synthetic._seed(6060, 9), 2048, 0.1), 64)
    srv = sb.Server(max_batch_molecules=4, max_batches=2, cycles_per_launch=25, **CONTROLS)
    ids = {}
    for k, m in enumerate(good):
        ids[srv.submit(m)] = ("minimize", m)
        ids[srv.submit(m, evaluate=True)] = ("evaluate", m)
        if k == 1:
            with pytest.raises(sb.StormmB200Error, match="Lennard-Jones type out of range"):
                srv.submit(bad_type)
            with pytest.raises(sb.StormmB200Error, match="exclusion partner out of range"):
                srv.submit(bad_excl, evaluate=True)
            bad_id = srv.submit(unbuildable, evaluate=True)
    assert srv.drain(120.0)
    results = srv.poll()
    st = srv.stats()
    srv.close()
    assert len(results) == len(ids) + 1
    assert st["failed"] == 1 and st["completed"] == len(ids) + 1 and st["in_flight"] == 0
    assert st["bytes_in_flight"] == 0.0 and st["batches"] == 0
    for r, arr in results:
        if r["request_id"] == bad_id:
            assert r["status"] != 0 and arr is None and np.isnan(r["energy"])
            continue
        assert r["status"] == 0
        kind, m = ids[r["request_id"]]
        if kind == "minimize":
            c_alone, e_alone, cyc_alone, _ = _alone(m)
            assert np.array_equal(arr, c_alone) and np.array_equal(r["energies"], e_alone)
            assert r["cycles"] == cyc_alone
        else:
            f_alone, e_alone = _evaluated_alone(m)
            assert np.array_equal(arr, f_alone) and np.array_equal(r["energies"], e_alone)


def test_fp64_server_minimizes_with_the_graph_kernel():
    """An FP64 server runs with the graph minimizer, and each result equals the FP64
    minimization of the molecule alone."""
    mols = [synthetic.make_molecule(synthetic._seed(6161, k), n, 0.3)
            for k, n in enumerate([24, 50, 81])]
    controls = dict(total_cycles=40, sd_cycles=10, convergence_rms=0.0, kernel=sb.MIN_GRAPH)
    opts = sb.default_options(precision=sb.PRECISION_DOUBLE)
    srv = sb.Server(cycles_per_launch=10, options=opts, **controls)
    ids = {srv.submit(m): m for m in mols}
    assert srv.drain(120.0)
    results = srv.poll()
    srv.close()
    assert len(results) == len(mols)
    for r, xyz in results:
        m = ids[r["request_id"]]
        syn = sb.Synthesis([m], options=sb.default_options(precision=sb.PRECISION_DOUBLE))
        syn.set_coordinates(m.coords)
        syn.minimize(**controls)
        assert r["status"] == 0
        assert np.array_equal(xyz, syn.coordinates())
        assert np.array_equal(r["energies"], syn.energies()[0])
        syn.close()


def test_emptying_batch_moves_its_molecules_to_waiting_requests():
    """Slot backfill: one batch at a time, four molecules a batch.  Three small molecules near
    a minimum converge within a few launches while a large, rough one keeps going; once they
    have retired, the large one moves with its minimizer state into a new batch beside the
    waiting requests and the first batch is released.  Every result is bit-identical to
    minimizing the molecule alone."""
    controls = dict(total_cycles=150, sd_cycles=30, convergence_rms=3.0, kernel=sb.MIN_PERSISTENT)
    mols = [synthetic.make_molecule(synthetic._seed(5150 + n, 0), n, 0.02) for n in (12, 14, 16)]
    mols.append(synthetic.make_molecule(synthetic._seed(5199, 0), 257, 0.5))
    mols += [synthetic.make_molecule(synthetic._seed(5151, k), n, 0.3)
             for k, n in enumerate([40, 48, 56, 64])]
    srv = sb.Server(max_batch_molecules=4, max_batches=1, cycles_per_launch=10, **controls)
    ids = {srv.submit(m): m for m in mols}
    assert srv.drain(120.0)
    results = srv.poll()
    st = srv.stats()
    srv.close()
    assert len(results) == len(mols) and st["failed"] == 0
    assert st["migrated"] >= 1
    assert st["admitted"] == len(mols) and st["bytes_in_flight"] == 0.0
    for r, xyz in results:
        m = ids[r["request_id"]]
        syn = sb.Synthesis([m])
        syn.set_coordinates(m.coords)
        syn.minimize(**controls)
        cycles, conv, _ = syn.minimize_progress()
        assert r["cycles"] == int(cycles[0]) and r["converged"] == bool(conv[0])
        assert np.array_equal(xyz, syn.coordinates().reshape(-1, 3))
        assert np.array_equal(r["energies"], syn.energies()[0])
        assert r["submit_time"] <= r["admit_time"] <= r["finish_time"]
        syn.close()
