"""STORMM's StaticExclusionMask tables from sb_static_exclusion_mask, bit for bit against the
tables STORMM built for every fixture (host code: runs without a GPU)."""
import os

import numpy as np
import pytest

import stormm_b200 as sb
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
