"""STORMM's own GPU path on the same B200: the comparison point for the evaluation and the minimizer.

TEST / MEASUREMENT INFRASTRUCTURE ONLY, used by bench.py's reference_gpu leg and by
tests/golden/make_gpu_minimizer_golden.py.  It runs oracle/_ref_gpu/stormm_gpu_driver, which
oracle/ref_gpu/Makefile builds from STORMM's sources with its CUDA path switched on, in a separate
process over Amber prmtop / inpcrd files of the molecules.  That process maps STORMM's library and
the CUDA runtime only; nothing of the package under test.

The driver's two modes (oracle/ref_gpu/gpu_driver.cpp):
  time      force + energy evaluations with launchNonbonded + launchValence over one
            AtomGraphSynthesis of all molecules, timed with CUDA events
  minimize  launchMinimization over the same synthesis, with energy histories
"""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref_gpu", "stormm_gpu_driver")
INPUT_ROOT = os.path.join(HERE, "_ref_gpu", "inputs")


def available() -> bool:
    return os.path.exists(DRIVER) and os.access(DRIVER, os.X_OK)


def read_records(path):
    """Records written by the drivers: name, dtype char, element count, raw data."""
    out = {}
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            n = struct.unpack("<i", h)[0]
            name = f.read(n).decode()
            dt = f.read(1).decode()
            cnt = struct.unpack("<q", f.read(8))[0]
            t = {"d": "<f8", "i": "<i4", "q": "<i8", "u": "<u4"}[dt]
            out[name] = np.frombuffer(f.read(cnt * np.dtype(t).itemsize), dtype=t).copy()
    return out


def write_inputs(tag: str, molecules) -> str:
    """Write the molecules as prmtop / inpcrd pairs under INPUT_ROOT/<tag> (once per tag) and
    return the list file the driver reads."""
    from stormm_b200 import prmtop
    d = os.path.join(INPUT_ROOT, tag)
    index = os.path.join(d, "index.txt")
    if os.path.exists(index):
        with open(index) as f:
            if sum(1 for line in f if line.strip()) == len(molecules):
                return index
    os.makedirs(d, exist_ok=True)
    lines = []
    for k, m in enumerate(molecules):
        top = os.path.join(d, f"m{k}.top")
        crd = os.path.join(d, f"m{k}.crd")
        prmtop.write_prmtop(m, top)
        prmtop.write_inpcrd(m, crd)
        lines.append(f"{top} {crd}\n")
    with open(index + ".tmp", "w") as f:
        f.writelines(lines)
    os.replace(index + ".tmp", index)
    return index


def _run(args, timeout):
    r = subprocess.run([DRIVER] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"STORMM GPU driver failed ({r.returncode}): "
                           f"{(r.stderr or r.stdout).strip()[-400:]}")
    line = [ln for ln in r.stdout.splitlines() if "=" in ln][-1]
    return {k: float(v) for k, v in (kv.split("=") for kv in line.split() if "=" in kv)}


def time_evaluations(list_file: str, evals: int, prec: str = "single", out: str | None = None,
                     timeout: float = 600.0) -> dict:
    """Time `evals` batched force + energy evaluations; value = systems x evals / second."""
    args = ["time", list_file, evals, "--prec", prec]
    if out:
        args += ["--out", out]
    f = _run(args, timeout)
    systems = int(f["systems"])
    return {"ms": f["ms"], "evals": int(f["evals"]), "systems": systems, "atoms": int(f["atoms"]),
            "ms_per_eval": f["ms"] / f["evals"],
            "value": systems * f["evals"] / (f["ms"] / 1000.0)}


def minimize(list_file: str, out: str, cycles: int, sd_cycles: int, ntpr: int = 1,
             prec: str = "single", clash_cycles: int = 0, clash_r0: float | None = None,
             clash_ratio: float | None = None, timeout: float = 1200.0) -> dict:
    """Run launchMinimization over the listed systems; returns the wall time of the call and
    the records (per-system potential-energy histories, final terms and coordinates)."""
    args = ["minimize", list_file, out, "--maxcyc", cycles, "--ncyc", sd_cycles, "--ntpr", ntpr,
            "--prec", prec]
    if clash_cycles > 0:
        args += ["--cdcyc", clash_cycles]
        if clash_r0 is not None:
            args += ["--clash-r0", clash_r0]
        if clash_ratio is not None:
            args += ["--clash-ratio", clash_ratio]
    f = _run(args, timeout)
    rec = read_records(out)
    lens = rec["min_history_length"]
    starts = np.concatenate([[0], np.cumsum(lens)])
    hist = [rec["min_potential_history"][starts[i]:starts[i + 1]] for i in range(len(lens))]
    return {"ms": f["ms"], "systems": int(f["systems"]), "atoms": int(f["atoms"]),
            "value": int(f["systems"]) / (f["ms"] / 1000.0), "histories": hist,
            "final_terms": rec["min_final_terms"].reshape(len(lens), -1),
            "start_coords": rec["min_start_coords"], "final_coords": rec["min_final_coords"]}
