"""sb_energies_to_host_static (energy export through the library's static scratch, no
allocation) against sb_get_energies on the same synthesis, on two calls in a row.  The file
name sorts last so the test also runs after every other test in one session."""
import ctypes

import numpy as np
import pytest

import stormm_b200 as sb
from stormm_b200 import synthetic

pytestmark = pytest.mark.gpu


def _entry():
    fn = sb.library().sb_energies_to_host_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_void_p]
    return fn


def test_static_export_matches_get_energies_twice():
    import torch
    fn = _entry()
    assert fn(None, 0, sb.NRG_STRIDE, 26, None, None) == sb.SB_OK   # per-device set-up
    mols = [synthetic.make_molecule(synthetic._seed(31337, k), n)
            for k, n in enumerate((24, 64, 100, 257))]
    syn = sb.Synthesis(mols)
    xyz = np.concatenate([m.coords for m in mols])
    rng = np.random.default_rng(5)
    for call in range(2):
        syn.set_coordinates(xyz + (0.0 if call == 0 else rng.normal(0.0, 0.02, xyz.shape)))
        syn.initialize()
        syn.evaluate()
        ref = syn.energies()
        dev = torch.from_numpy(syn.energies_fixed().reshape(-1).copy()).cuda()
        torch.cuda.synchronize()
        out = np.full(syn.nsys * sb.NRG_STRIDE, np.nan)
        rc = fn(dev.data_ptr(), syn.nsys, sb.NRG_STRIDE, 26, out.ctypes.data, None)
        assert rc == sb.SB_OK, sb.library().sb_last_error()
        np.testing.assert_allclose(out.reshape(syn.nsys, sb.NRG_STRIDE), ref, rtol=1e-12,
                                   atol=1e-12)
    syn.close()


def test_static_export_rejects_oversized_requests():
    fn = _entry()
    out = np.zeros(16)
    rc = fn(None, 4097, sb.NRG_STRIDE, 26, out.ctypes.data, None)
    assert rc == -1
    assert b"static scratch" in sb.library().sb_last_error()
