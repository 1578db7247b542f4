"""Surface area (STORMM's sphere-point SASA of its MM-GBSA application).

Fixtures (tests/golden/make_golden.py --sasa-only): three synthetic molecules (60, 200 and 33
atoms; 272, 272 and 100 sphere points) with STORMM's points, area and energy.  The CPU
restatement in the oracle matches STORMM to 1e-10 relative (same point verdicts; only the order
of the sum differs); the GPU kernel (sb_surface_area) matches STORMM the same way, alone and in a
batch."""
import numpy as np
import pytest

import oracle
from fixtures import load, molecule_from_fixture

CASES = ["sasa_s60.npz", "sasa_s200.npz", "sasa_s33.npz"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_surface_area_matches_stormm(name):
    g = load(name)
    m = molecule_from_fixture(g)
    area = oracle.surface_area(g["coords"].reshape(-1, 3), oracle.sasa_radii(m),
                               g["sphere_points"])
    assert abs(area - g["sasa_area"][0]) <= 1e-10 * g["sasa_area"][0]
    energy = oracle.surface_area(g["coords"].reshape(-1, 3), oracle.sasa_radii(m),
                                 g["sphere_points"], weight=0.005)
    assert abs(energy - g["sasa_energy"][0]) <= 1e-10 * g["sasa_energy"][0]


@pytest.mark.gpu
def test_gpu_surface_area_matches_stormm_alone_and_batched():
    import stormm_b200 as sb
    gs = [load(n) for n in CASES]
    mols = [molecule_from_fixture(g) for g in gs]
    batch = sb.Synthesis(mols)
    batch.set_coordinates(np.concatenate([m.coords for m in mols]))
    for k, (g, m) in enumerate(zip(gs, mols)):
        syn = sb.Synthesis([m])
        syn.set_coordinates(m.coords)
        area = syn.surface_area(g["sphere_points"])[0]
        assert abs(area - g["sasa_area"][0]) <= 1e-10 * g["sasa_area"][0], (k, area)
        energy = syn.surface_area(g["sphere_points"], weight=0.005)[0]
        assert abs(energy - g["sasa_energy"][0]) <= 1e-10 * g["sasa_energy"][0]
        assert batch.surface_area(g["sphere_points"])[k] == area
        syn.close()
    with pytest.raises(sb.StormmB200Error):
        batch.surface_area(np.zeros((0, 3)))
    batch.close()
