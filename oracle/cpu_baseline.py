"""Timed CPU baseline: STORMM's own CPU evaluators on the host cores.

TEST / BASELINE INFRASTRUCTURE ONLY, used by bench.py's CPU-baseline leg and reference arm.

STORMM's CPU path is single-threaded FP64 (MolecularMechanics/mm_evaluation.tpp:630,
evalRestrainedMMGB; minimize() for minimization), so the baseline runs one process per host
core on disjoint shards of a bounded sample of the workload and reports the aggregate.  When the
reference build (oracle/_ref/stormm_ref_driver) is absent, the FP64 C restatement in this
directory stands in, with the same process-per-core layout.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import subprocess
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "stormm_ref_driver")


def reference_available() -> bool:
    return os.path.exists(DRIVER) and os.access(DRIVER, os.X_OK)


def _write_shards(molecules, nproc, tmpdir):
    from stormm_b200 import prmtop
    lists = []
    for p in range(nproc):
        path = os.path.join(tmpdir, f"shard{p}.txt")
        with open(path, "w") as f:
            for k in range(p, len(molecules), nproc):
                m = molecules[k]
                top = os.path.join(tmpdir, f"m{k}.top")
                crd = os.path.join(tmpdir, f"m{k}.crd")
                if not os.path.exists(top):
                    prmtop.write_prmtop(m, top)
                    prmtop.write_inpcrd(m, crd)
                f.write(f"{top} {crd}\n")
        lists.append(path)
    return lists


def _port_worker(args):
    """Evaluate molecules with the FP64 oracle for a fixed wall time (one process)."""
    idx, seconds, minimize_cycles, sd_cycles, seed_list = args
    import oracle
    from stormm_b200 import synthetic
    mols = [synthetic.make_molecule(s, n, noise=nz) for (s, n, nz) in seed_list]
    systems = [oracle.from_molecule(m) for m in mols]
    t0 = time.perf_counter()
    count = 0
    k = 0
    while time.perf_counter() - t0 < seconds:
        if minimize_cycles > 0:
            systems[k].minimize(mols[k].coords, minimize_cycles, sd_cycles)
        else:
            systems[k].evaluate(mols[k].coords)
        count += 1
        k = (k + 1) % len(systems)
    return count, time.perf_counter() - t0


def run(molecules, seconds: float = 10.0, nproc: int | None = None, minimize_cycles: int = 0,
        molecule_seeds=None, sd_cycles: int = 50):
    """Aggregate evaluations (or minimizations) per second of the CPU baseline.

    molecules: the bounded sample (Molecule objects).  molecule_seeds: optional list of
    (seed, natom, noise) that rebuilds the same sample, needed only by the port fallback.
    Returns a dict with value, unit, cores, kind, sample."""
    nproc = nproc or os.cpu_count() or 1
    nproc = max(1, min(nproc, len(molecules)))
    what = "minimizations" if minimize_cycles > 0 else "evals"
    if reference_available():
        with tempfile.TemporaryDirectory() as tmp:
            lists = _write_shards(molecules, nproc, tmp)
            extra = (["--minimize", str(minimize_cycles), "--ncyc", str(sd_cycles)]
                     if minimize_cycles > 0 else [])
            procs = [subprocess.Popen([DRIVER, "time", lst, str(seconds)] + extra,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
                     for lst in lists]
            total, tmax = 0, 0.0
            for p in procs:
                out, err = p.communicate()
                if p.returncode != 0:
                    raise RuntimeError(f"reference CPU driver failed: {err.strip()[-400:]}")
                fields = dict(kv.split("=") for kv in out.split())
                total += int(fields[what])
                tmax = max(tmax, float(fields["seconds"]))
        kind = "reference"
    else:
        if molecule_seeds is None:
            raise RuntimeError("reference CPU build missing and no seeds for the oracle port")
        ctx = mp.get_context("spawn")
        shards = [molecule_seeds[p::nproc] for p in range(nproc)]
        with ctx.Pool(nproc) as pool:
            res = pool.map(_port_worker, [(p, seconds, minimize_cycles, sd_cycles, shards[p])
                                          for p in range(nproc)])
        total = sum(r[0] for r in res)
        tmax = max(r[1] for r in res)
        kind = "port"
    return {"value": total / tmax, "unit": f"{'minimizations' if minimize_cycles else 'force-evals'}/s",
            "cores": nproc, "kind": kind, "count": total, "seconds": tmax}
