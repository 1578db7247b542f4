"""The STORMM-named C++ layer (include/stormm_b200.hpp) through a compiled caller,
tests/cpp/launcher_check.cpp.

Host: the program compiles against the header and links the library; topology and coordinate
reading, synthesis set-up and the error behaviour (std::runtime_error with the library's message)
work without a device.  Device: launchValence + launchNonbonded into a ScoreCard, a clash-damped
energy-only launchNonbonded, and launchMinimization give bit for bit what the same operations
give through the Python binding (the same kernels behind one C ABI), and the energies and forces
agree with the FP64 oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
import stormm_b200 as sb
from stormm_b200 import prmtop as amber_writer
from stormm_b200 import synthetic

from conftest import ROOT
from fixtures import check_energies, oracle_magnitudes, rms_rel

SOURCE = os.path.join(ROOT, "tests", "cpp", "launcher_check.cpp")
LIBDIR = os.path.join(ROOT, "stormm_b200")


def _compile(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "launcher_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
           os.path.join(ROOT, "include"), SOURCE, "-o", exe, "-L", LIBDIR, "-lstormm_b200",
           f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _parse(path):
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if parts[0] == "error":
                out.setdefault("errors", {})[parts[1]] = (parts[2] == "1", " ".join(parts[3:]))
                continue
            if parts[0] == "upload":
                out["upload"] = parts[2] == "1"
                continue
            n = int(parts[1])
            out[parts[0]] = np.array([float(v) for v in parts[2:2 + n]])
    return out


def _write(tmp_path, mols):
    files = []
    for k, m in enumerate(mols):
        top, crd = str(tmp_path / f"m{k}.prmtop"), str(tmp_path / f"m{k}.inpcrd")
        amber_writer.write_prmtop(m, top)
        amber_writer.write_inpcrd(m, crd)
        files += [top, crd]
    return files


def test_header_compiles_and_host_paths_work(tmp_path):
    exe = _compile(tmp_path)
    mol = synthetic.make_molecule(seed=21, natom=30)
    files = _write(tmp_path, [mol])
    out_path = str(tmp_path / "host.txt")
    r = subprocess.run([exe, "host", out_path] + files, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = _parse(out_path)
    assert int(out["atoms"][0]) == 30 and int(out["systems"][0]) == 2
    np.testing.assert_allclose(out["coords"].reshape(-1, 3),
                               sb.read_amber_coordinates(files[1], 30), rtol=0, atol=0)
    abstracts, insr = sb.nonbonded_work_units([mol], np.array([0, 0]), init_task=3)
    np.testing.assert_array_equal(out["nbwu_abstracts"], abstracts.reshape(-1))
    np.testing.assert_array_equal(out["nbwu_insr"], insr.reshape(-1))
    for label, (ok, msg) in out["errors"].items():
        assert ok, (label, msg)
    assert set(out["errors"]) == {"missing_file", "empty_scorecard", "topology_index",
                                  "launch_before_upload", "minimize_controls"}


@pytest.mark.gpu
def test_launchers_match_python_path_and_oracle(tmp_path):
    exe = _compile(tmp_path)
    src = [synthetic.make_molecule(seed=31, natom=24), synthetic.make_molecule(seed=32, natom=90),
           synthetic.make_chain(seed=33, natom=150)]
    files = _write(tmp_path, src)
    out_path = str(tmp_path / "device.txt")
    r = subprocess.run([exe, "device", out_path] + files, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    cpp = _parse(out_path)

    mols = [sb.read_amber(files[2 * k], files[2 * k + 1], igb=sb.SB_GB_OBC2)
            for k in range(len(src))]
    index = [0, 1, 2, 0, 1, 2]
    nsys = len(index)
    xyz = np.concatenate([mols[t].coords for t in index])
    syn = sb.Synthesis(mols, topology_index=index, igb=sb.SB_GB_OBC2)
    syn.set_coordinates(xyz)
    syn.initialize()
    syn.evaluate(terms=sb.TERM_VALENCE)
    syn.evaluate(terms=sb.TERM_NONBONDED | sb.TERM_GB)
    energies = syn.energies()
    forces = syn.forces()
    psi, radii, _ = syn.gb_workspace()
    assert syn.status() == 0
    # identical kernels behind both bindings: bit for bit
    np.testing.assert_array_equal(cpp["energies"], energies.reshape(-1))
    np.testing.assert_array_equal(cpp["forces"], forces.reshape(-1))
    np.testing.assert_array_equal(cpp["psi"], psi.reshape(-1))
    np.testing.assert_array_equal(cpp["radii"], radii.reshape(-1))
    np.testing.assert_allclose(cpp["potential"], energies.reshape(nsys, -1)[:, :13].sum(axis=1),
                               rtol=1e-14, atol=1e-9)

    # and both agree with the FP64 oracle on the files' topologies
    e = cpp["energies"].reshape(nsys, sb.NRG_STRIDE)
    f = cpp["forces"].reshape(-1, 3)
    off = 0
    for s, t in enumerate(index):
        m = mols[t]
        o = oracle.from_molecule(m, igb=sb.SB_GB_OBC2).evaluate(m.coords)
        got = np.array([e[s, sb.NRG_SLOTS[k]] for k in sb.TERM_ORDER])
        check_energies(got, o["energies"], oracle_magnitudes(m), s)
        assert rms_rel(f[off:off + m.natom], o["forces"]) <= 5e-6
        off += m.natom

    # clash-damped, energy-only nonbonded launch
    syn.initialize(sb.INIT_ENERGIES)
    syn.evaluate_clash(0.5, 0.8, terms=sb.TERM_NONBONDED | sb.TERM_GB, force=False)
    np.testing.assert_array_equal(cpp["clash_energies"], syn.energies().reshape(-1))

    # launchMinimization: 40 cycles, 10 of steepest descent, 5 clash-damped, every cycle run
    syn.set_coordinates(xyz)
    syn.minimize(total_cycles=40, sd_cycles=10, clash_cycles=5, clash_distance=0.2,
                 clash_ratio=0.5, convergence_rms=0.0, record_history=1)
    fin = syn.energies().reshape(nsys, -1)
    np.testing.assert_allclose(cpp["min_potential"], fin[:, :13].sum(axis=1), rtol=1e-14,
                               atol=1e-9)
    np.testing.assert_array_equal(cpp["min_coords"], syn.coordinates().reshape(-1))
    hist = syn.minimize_history()
    samples = np.concatenate([np.append(hist[s, 0:40:10], hist[s, 40]) for s in range(nsys)])
    np.testing.assert_array_equal(cpp["min_history"], samples)
    assert np.all(cpp["min_potential"] < cpp["potential"])

    # the line search step by step through launchConjugateGradient / launchLineAdvance, against
    # the same steps through the C ABI from Python; the C++ caller starts from the coordinates its
    # PhaseSpaceSynthesis downloaded after launchMinimization
    syn.set_coordinates(cpp["min_coords"])
    syn.minimize_begin(total_cycles=12, sd_cycles=4, clash_cycles=0, convergence_rms=0.0,
                       kernel=sb.MIN_GRAPH)
    for _ in range(12):
        for move in range(4):
            syn.initialize(sb.INIT_ENERGIES | (sb.INIT_FORCES if move == 0 else 0))
            syn.launch_valence(force=(move == 0))
            syn.launch_nonbonded(force=(move == 0))
            if move == 0:
                syn.conjugate_gradient()
            syn.line_advance(move)
    np.testing.assert_array_equal(cpp["steps_coords"], syn.coordinates().reshape(-1))

    # PrecisionModel::DOUBLE: the same minimization on a synthesis uploaded for FP64
    syn64 = sb.Synthesis(mols, topology_index=index, igb=sb.SB_GB_OBC2,
                         precision=sb.PRECISION_DOUBLE)
    syn64.set_coordinates(xyz)
    syn64.minimize(total_cycles=40, sd_cycles=10, clash_cycles=5, clash_distance=0.2,
                   clash_ratio=0.5, convergence_rms=0.0, kernel=sb.MIN_GRAPH)
    np.testing.assert_array_equal(cpp["min64_coords"], syn64.coordinates().reshape(-1))
    fin64 = syn64.energies().reshape(nsys, -1)
    np.testing.assert_allclose(cpp["min64_potential"], fin64[:, :13].sum(axis=1), rtol=1e-14,
                               atol=1e-9)
