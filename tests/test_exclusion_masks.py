"""STORMM's StaticExclusionMask tables from sb_static_exclusion_mask, bit for bit against the
tables STORMM built for every fixture (host code: runs without a GPU)."""
import glob
import os

import numpy as np
import pytest

import stormm_b200 as sb
from conftest import GOLDEN
from fixtures import load, molecule_from_fixture, reference_paths, synthetic_paths


@pytest.mark.parametrize("path", synthetic_paths() + reference_paths(), ids=os.path.basename)
def test_static_exclusion_mask_is_bit_exact(path):
    g = load(os.path.basename(path))
    if "se_mask_data" not in g:
        pytest.skip("fixture without exclusion tables")
    out = sb.static_exclusion_mask(molecule_from_fixture(g))
    assert out["supertile_stride_count"] == int(g["se_supertile_stride_count"][0])
    assert np.array_equal(out["supertile_map_idx"], g["se_supertile_map_idx"])
    assert np.array_equal(out["tile_map_idx"], g["se_tile_map_idx"])
    assert np.array_equal(out["mask_data"], g["se_mask_data"].astype(np.uint32))


def test_static_exclusion_mask_rejects_small_outputs():
    g = load("synthetic_E100.npz")
    import ctypes
    t = sb._TopologyArrays(molecule_from_fixture(g))
    sup = np.zeros(1, dtype=np.int32)
    n = [ctypes.c_longlong(1), ctypes.c_longlong(0), ctypes.c_longlong(0)]
    nst = ctypes.c_int()
    rc = sb.library().sb_static_exclusion_mask(ctypes.byref(t.struct), ctypes.byref(nst),
                                               sup.ctypes.data, ctypes.byref(n[0]), None,
                                               ctypes.byref(n[1]), None, ctypes.byref(n[2]))
    assert rc == sb.SB_OK      # a 100-atom system has one supertile: one entry fits
    n[0] = ctypes.c_longlong(0)
    rc = sb.library().sb_static_exclusion_mask(ctypes.byref(t.struct), ctypes.byref(nst),
                                               sup.ctypes.data, ctypes.byref(n[0]), None,
                                               ctypes.byref(n[1]), None, ctypes.byref(n[2]))
    assert rc == -1


def _nbwu_case(path):
    from stormm_b200 import synthetic
    g = load(os.path.basename(path))
    mols = []
    for gen, seed, n in zip(g["generators"], g["seeds"], g["natoms"]):
        make = synthetic.make_chain if str(gen) == "chain" else synthetic.make_molecule
        mols.append(make(int(seed), int(n)))
    return g, mols


def _same(g, key, got):
    import hashlib
    if key in g:
        return np.array_equal(got, g[key].astype(got.dtype))
    return (got.size == int(g[key + "_size"][0]) and
            hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() ==
            str(g[key + "_sha256"][0]))


NBWU_PATHS = sorted(glob.glob(os.path.join(GOLDEN, "nbwu_*.npz")))


@pytest.mark.parametrize("path", NBWU_PATHS, ids=os.path.basename)
def test_static_exclusion_mask_synthesis_is_bit_exact(path):
    """The synthesis-level mask tables (topologies shared by several systems, indices shifted
    past earlier topologies' tables) equal STORMM's StaticExclusionMaskSynthesis."""
    g, mols = _nbwu_case(path)
    ms = sb.static_exclusion_mask_synthesis(mols, g["index"])
    for key in ("supertile_map_bounds", "supertile_map_idx", "tile_map_idx", "mask_data"):
        assert _same(g, "se_" + key, ms[key]), key


@pytest.mark.parametrize("path", NBWU_PATHS, ids=os.path.basename)
def test_nonbonded_work_units_are_bit_exact(path):
    """STORMM's nonbonded work units (8-, 16-, 32- and 64-tile targets, the import-limit
    backtracking, initialization masks and refresh ranges of several InitializationTasks):
    abstracts and tile instructions equal AtomGraphSynthesis::loadNonbondedWorkUnits'."""
    g, mols = _nbwu_case(path)
    abstracts, insr = sb.nonbonded_work_units(mols, g["index"], init_task=int(g["init_task"][0]))
    assert _same(g, "nbwu_abstracts", abstracts.reshape(-1))
    assert _same(g, "nbwu_insr", insr.reshape(-1))
    # every tile of every system appears once
    n_tiles = sum(((int(n) + 15) // 16) * ((int(n) + 15) // 16 + 1) // 2 * int(c)
                  for n, c in zip(g["natoms"], g["counts"]))
    assert int((abstracts[:, 27] - abstracts[:, 26]).sum()) == n_tiles


def test_nonbonded_work_units_refuse_huge_syntheses():
    from stormm_b200 import synthetic
    big = synthetic.make_chain(4601, 5000)
    with pytest.raises(sb.StormmB200Error, match="256-tile"):
        sb.nonbonded_work_units([big], np.zeros(200, dtype=np.int32))


def test_work_unit_and_mask_synthesis_argument_checks():
    from stormm_b200 import synthetic
    m = synthetic.make_molecule(4701, 40)
    with pytest.raises(sb.StormmB200Error, match="initialization task"):
        sb.nonbonded_work_units([m], [0], init_task=9)
    with pytest.raises(sb.StormmB200Error, match="out of range"):
        sb.nonbonded_work_units([m], [1])
    with pytest.raises(sb.StormmB200Error, match="out of range"):
        sb.static_exclusion_mask_synthesis([m], [0, 2])
    # a synthesis of one system reproduces the single-topology tables
    one = sb.static_exclusion_mask(m)
    syn = sb.static_exclusion_mask_synthesis([m], [0])
    assert np.array_equal(syn["supertile_map_idx"], one["supertile_map_idx"])
    assert np.array_equal(syn["tile_map_idx"], one["tile_map_idx"])
    assert np.array_equal(syn["mask_data"], one["mask_data"])
