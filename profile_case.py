"""Small, fixed profiling cases for the evaluation and minimization kernels.

  python profile_case.py [--molecules 256] [--evals 4] [--energy-only]
  python profile_case.py --workload minimization --molecules 4096 --minimize 20
  python profile_case.py --workload chains --molecules 16 --evals 3
  python profile_case.py --workload chains --molecules 16 --evals 3 --precision double

The first form builds the first molecules of the batched single-point workload (16-256 atoms),
uploads them and runs a few force + energy evaluations; the second builds the first molecules
of the minimization workload (24-96 atoms, 0.3 A noise) and runs a short minimization; the third
evaluates the first chains of the large-system workload (2,000-5,000 atoms, tiled path).  All
finish in seconds, so a profiler can capture single launches of each kernel.
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="single-point",
                    choices=["single-point", "minimization", "chains"])
    ap.add_argument("--molecules", type=int, default=256)
    ap.add_argument("--evals", type=int, default=4)
    ap.add_argument("--energy-only", action="store_true")
    ap.add_argument("--minimize", type=int, default=0, help="minimization cycles")
    ap.add_argument("--precision", default="single", choices=["single", "double"])
    args = ap.parse_args()
    import stormm_b200 as sb
    from stormm_b200 import synthetic
    if args.workload == "minimization":
        mols = synthetic.workload_minimization(args.molecules)
    elif args.workload == "chains":
        mols = synthetic.workload_chains(args.molecules)
    else:
        mols = synthetic.workload_batched_single_point(args.molecules)
    syn = sb.Synthesis(mols, precision=(sb.PRECISION_DOUBLE if args.precision == "double"
                                        else sb.PRECISION_SINGLE))
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    if args.minimize > 0:
        syn.minimize(total_cycles=args.minimize, sd_cycles=min(50, args.minimize))
    else:
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
