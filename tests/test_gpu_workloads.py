"""The timed workloads themselves, at full size, against the FP64 oracle and STORMM's own CPU
results, through the C ABI.

* batched single point: all 1,024 molecules of 16-256 atoms (OBC-II), every molecule's energy
  terms and forces against the FP64 oracle under the bounds of tests/fixtures.py, and a
  64-molecule sample (every 16th) against STORMM's own CPU build
  (tests/golden/workload_single_point_sample.npz, made by make_workload_golden.py);
* the same 1,024 molecules in the FP64 mode (PrecisionModel::DOUBLE): every term within 1e-6 of
  max(|E_term|, 1 kcal/mol), without the root-sum-square scale, forces to 5e-6;
* batched minimization: all 4,096 molecules of 24-96 atoms (0.3 A start noise), the start
  evaluation of every molecule against the oracle, then the first line-minimization cycle of the
  graph minimizer against the oracle's restatement of STORMM's GPU line search: the energy after
  the cycle within 1e-5 relative (the single-cycle bound of tests/test_gpu_minimize.py: the
  move follows the FP32 forces, which carry up to 5e-6 RMS relative error).
"""
import os

import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from stormm_b200 import synthetic
from conftest import GOLDEN
from fixtures import FORCE_TOL, check_energies, rms_rel, total_tolerance

pytestmark = pytest.mark.gpu


def _reference(mols, coords=None):
    """Oracle energies, forces and per-term root-sum-squares of every molecule."""
    out = []
    for k, m in enumerate(mols):
        c = m.coords if coords is None else coords[k]
        osys = oracle.from_molecule(m)
        r = osys.evaluate(c)
        r["rss"] = osys.magnitudes(c, r["radii"])
        out.append(r)
    return out


@pytest.fixture(scope="module")
def single_point():
    mols = synthetic.workload_batched_single_point(1024, seed=synthetic.SEED_BASE + 1)
    return mols, _reference(mols)


def _evaluate(mols, coords, **opts):
    syn = sb.Synthesis(mols, **opts)
    syn.set_coordinates(np.concatenate(coords))
    syn.initialize()
    syn.evaluate()
    assert syn.status() == 0
    out = syn.energy_terms(), syn.split(syn.forces())
    syn.close()
    return out


def test_full_single_point_workload_matches_oracle(single_point):
    mols, ref = single_point
    energies, forces = _evaluate(mols, [m.coords for m in mols])
    for k, m in enumerate(mols):
        check_energies(energies[k], ref[k]["energies"], ref[k]["rss"], (k, m.natom))
        assert rms_rel(forces[k], ref[k]["forces"]) <= FORCE_TOL, (k, m.natom)


def test_full_single_point_workload_fp64_mode_meets_the_plain_bound(single_point):
    mols, ref = single_point
    energies, forces = _evaluate(mols, [m.coords for m in mols], precision=sb.PRECISION_DOUBLE)
    for k, m in enumerate(mols):
        check_energies(energies[k], ref[k]["energies"], None, (k, m.natom))
        assert rms_rel(forces[k], ref[k]["forces"]) <= FORCE_TOL, (k, m.natom)


def test_single_point_sample_matches_stormm_cpu_build():
    """64 molecules of the workload against STORMM's evalRestrainedMMGB and per-term FP64
    evaluators at the coordinates STORMM used (rounded to the 2^-32 A grid)."""
    g = dict(np.load(os.path.join(GOLDEN, "workload_single_point_sample.npz")))
    allmols = synthetic.workload_batched_single_point(1024, seed=synthetic.SEED_BASE + 1)
    mols = [allmols[k] for k in g["index"]]
    offs = np.concatenate([[0], np.cumsum(g["natom"])])
    coords = [g["coords"][offs[j]:offs[j + 1]] for j in range(len(mols))]
    energies, forces = _evaluate(mols, coords)
    for j, m in enumerate(mols):
        assert m.natom == g["natom"][j]
        rss = oracle.from_molecule(m).magnitudes(coords[j])
        check_energies(energies[j], g["energy_terms"][j], rss, (int(g["index"][j]), m.natom))
        assert rms_rel(forces[j], g["forces"][offs[j]:offs[j + 1]]) <= FORCE_TOL, j


def test_minimization_workload_first_cycle_matches_oracle():
    mols = synthetic.workload_minimization(4096, seed=synthetic.SEED_BASE + 2)
    ref = _reference(mols)
    energies, forces = _evaluate(mols, [m.coords for m in mols])
    for k, m in enumerate(mols):
        check_energies(energies[k], ref[k]["energies"], ref[k]["rss"], (k, m.natom))
        assert rms_rel(forces[k], ref[k]["forces"]) <= FORCE_TOL, (k, m.natom)
    syn = sb.Synthesis(mols)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    syn.minimize(total_cycles=1, sd_cycles=50, record_history=True, kernel=sb.MIN_GRAPH)
    assert syn.status() == 0
    hist = syn.minimize_history()
    syn.close()
    for k, m in enumerate(mols):
        _, h_ref = oracle.from_molecule(m).minimize(m.coords, 1, 50)
        assert abs(hist[k, 0] - h_ref[0]) <= total_tolerance(ref[k]["energies"], ref[k]["rss"])
        assert abs(hist[k, 1] - h_ref[1]) <= 1e-5 * abs(h_ref[1]), (k, hist[k], h_ref)
        assert hist[k, 1] < hist[k, 0]
