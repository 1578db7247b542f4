"""The C-ABI library loads and exports every entry point include/stormm_b200.h declares.  These
checks make no compute call, so they run without a GPU."""
import ctypes
import os
import re

import pytest

import stormm_b200
from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "stormm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "sb_synthesis_create" in names and "sb_evaluate" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = stormm_b200.library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared but not exported: {missing}"


def test_version_and_defaults_without_gpu():
    lib = stormm_b200.library()
    assert b"sm_100a" in lib.sb_version()
    o = stormm_b200.default_options()
    assert o.igb == 5 and o.dielectric == 80.0 and o.frc_bits == 23 and o.gpos_bits == 32


def test_null_handle_is_an_error():
    lib = stormm_b200.library()
    rc = lib.sb_evaluate(None, 7, 1, 1, None)
    assert rc == -1
    assert b"null" in lib.sb_last_error()


def test_server_checks_its_controls_on_the_host():
    """The request server refuses bad minimization controls and an FP64 server without the
    graph minimizer when it is created, before any device is touched."""
    with pytest.raises(stormm_b200.StormmB200Error, match="initial step"):
        stormm_b200.Server(initial_step=-1.0)
    with pytest.raises(stormm_b200.StormmB200Error, match="clash-damping"):
        stormm_b200.Server(clash_cycles=5, clash_distance=-0.2)
    with pytest.raises(stormm_b200.StormmB200Error, match="graph minimizer"):
        stormm_b200.Server(options=stormm_b200.default_options(
            precision=stormm_b200.PRECISION_DOUBLE), kernel=stormm_b200.MIN_PERSISTENT)


def test_served_result_layout_matches_the_header():
    """The Python mirror of sb_served_result and sb_server_stats has the C layout."""
    r = stormm_b200.ServedResult
    assert r.status.offset == 24 and r.rms_force.offset == 32
    assert ctypes.sizeof(r) == 32 + 8 + 8 + 8 * 16 + 3 * 8
    assert stormm_b200.ServerStats.failed.offset == 24
    assert stormm_b200.ServerStats.migrated.offset == 32


def test_server_options_default_and_checks():
    """sb_default_server_options sets every field (the migration threshold included), and the
    server refuses a migration threshold outside [0, 1)."""
    o = stormm_b200.ServerOptions()
    stormm_b200.library().sb_default_server_options(ctypes.byref(o))
    assert o.migrate_fraction == 0.25 and o.cycles_per_launch == 50
    assert stormm_b200.ServerOptions.migrate_fraction.offset == (
        stormm_b200.ServerOptions.cycles_per_launch.offset + 8)
    for bad in (-0.1, 1.0):
        with pytest.raises(stormm_b200.StormmB200Error, match="migrate_fraction"):
            stormm_b200.Server(migrate_fraction=bad)
