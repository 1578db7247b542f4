"""Generate tests/golden/gpu_minimize_<case>.npz by running STORMM's own GPU line minimizer.

Requires a GPU and the reference CUDA build (oracle/ref_gpu/Makefile:
oracle/_ref_gpu/stormm_gpu_driver).  Run from the repository root:

    python tests/golden/make_gpu_minimizer_golden.py [output directory]

The molecules (MOLECULES: seeded synthetic molecules of 24-200 atoms, 0.3 A start noise) are
written as Amber prmtop / inpcrd files, read by STORMM's AtomGraph / PhaseSpace and minimized
together in one synthesis by launchMinimization (MolecularMechanics/hpc_minimization.h:138),
OBC-II GB, CYCLES line-minimization cycles of which SD_CYCLES steepest descent, one energy
sample per cycle.  The cases (CASES) cover STORMM's FP32 and FP64 precision models, plain and
with the first CLASH_CYCLES cycles clash-damped.  Each fixture keeps the molecules' seeds and
sizes, the coordinates STORMM started from (on its 2^-32 A grid), the potential energy at the
start of every cycle and at the end, the final per-term energies and the final coordinates.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import gpu_reference  # noqa: E402
from stormm_b200 import synthetic  # noqa: E402

SEED = 5150
SIZES = [24, 31, 40, 48, 57, 64, 72, 80, 88, 96, 128, 200]
NOISE = 0.3
CYCLES = 200
SD_CYCLES = 50
CLASH_CYCLES = 25
CLASH_DISTANCE = 0.2
CLASH_RATIO = 0.5
CASES = {
    "fp32": dict(prec="single", clash_cycles=0),
    "fp32_clash": dict(prec="single", clash_cycles=CLASH_CYCLES),
    "fp64": dict(prec="double", clash_cycles=0),
    "fp64_clash": dict(prec="double", clash_cycles=CLASH_CYCLES),
}


def molecules():
    return [synthetic.make_molecule(synthetic._seed(SEED, k), n, noise=NOISE, name=f"G{k}")
            for k, n in enumerate(SIZES)]


def main(outdir: str) -> None:
    if not gpu_reference.available():
        raise SystemExit("reference CUDA build missing: make -C oracle/ref_gpu")
    os.makedirs(outdir, exist_ok=True)
    mols = molecules()
    with tempfile.TemporaryDirectory() as tmp:
        gpu_reference.INPUT_ROOT = tmp
        lst = gpu_reference.write_inputs("gpu_minimizer", mols)
        for case, kw in CASES.items():
            clash = kw["clash_cycles"] > 0
            r = gpu_reference.minimize(lst, os.path.join(tmp, case + ".bin"), CYCLES, SD_CYCLES,
                                       ntpr=1, prec=kw["prec"], clash_cycles=kw["clash_cycles"],
                                       clash_r0=CLASH_DISTANCE if clash else None,
                                       clash_ratio=CLASH_RATIO if clash else None)
            hist = np.stack(r["histories"])
            out = os.path.join(outdir, f"gpu_minimize_{case}.npz")
            np.savez_compressed(out, seed=SEED, sizes=np.array(SIZES), noise=NOISE,
                                cycles=CYCLES, sd_cycles=SD_CYCLES,
                                clash_cycles=kw["clash_cycles"], clash_distance=CLASH_DISTANCE,
                                clash_ratio=CLASH_RATIO, precision=kw["prec"],
                                start_coords=r["start_coords"], history=hist,
                                final_terms=r["final_terms"], final_coords=r["final_coords"])
            print(f"{case}: {len(SIZES)} molecules, {hist.shape[1]} samples, "
                  f"E0 {hist[:, 0].sum():.4f} -> {hist[:, -1].sum():.4f}, "
                  f"{r['ms']:.1f} ms -> {out}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
