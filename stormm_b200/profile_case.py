"""Small, fixed profiling case for the fused evaluation kernel.

  python -m stormm_b200.profile_case [--molecules 256] [--evals 4] [--energy-only]

Builds the first molecules of the batched single-point workload (16-256 atoms), uploads them and
runs a few force + energy evaluations, so a profiler can capture single launches of the kernel
on a case that finishes in seconds.
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecules", type=int, default=256)
    ap.add_argument("--evals", type=int, default=4)
    ap.add_argument("--energy-only", action="store_true")
    args = ap.parse_args()
    import stormm_b200 as sb
    from stormm_b200 import synthetic
    mols = synthetic.workload_batched_single_point(args.molecules)
    syn = sb.Synthesis(mols)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    for _ in range(args.evals):
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate(force=not args.energy_only, energy=True)
    e = syn.energy_terms()
    if syn.status() != 0:
        raise SystemExit("device status word set")
    print("profile case done:", args.molecules, "molecules, total energy", float(e.sum()))
    syn.close()


if __name__ == "__main__":
    main()
