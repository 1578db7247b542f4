"""Timed CPU baseline: STORMM's own CPU evaluators on the host cores.

TEST / BASELINE INFRASTRUCTURE ONLY, used by bench.py's CPU-baseline leg and reference arm.

STORMM's CPU path is single-threaded FP64 (MolecularMechanics/mm_evaluation.tpp:630,
evalRestrainedMMGB; minimize() for minimization), so the baseline runs one process per host
core on disjoint shards of a bounded sample of the workload and reports the aggregate.  When the
reference build (oracle/_ref/stormm_ref_driver) is absent, the FP64 C restatement in this
directory stands in, with the same process-per-core layout.

The samples are the leading molecules of the benchmark workloads (SAMPLES).  prepare_samples()
writes them once as Amber prmtop / inpcrd files under oracle/_ref/samples/ (the build step does
this where the reference build exists), so that a timed run reads STORMM's own inputs and maps
no library of the package under test.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "stormm_ref_driver")
SAMPLE_ROOT = os.path.join(HERE, "_ref", "samples")

# name: (workload, molecules in the sample, minimization cycles, steepest-descent cycles)
SAMPLES = {
    "single_point": ("batched_single_point", 256, 0, 0),
    "minimization": ("minimization", 128, 500, 50),
    "large": ("chains", 16, 0, 0),
}


def reference_available() -> bool:
    return os.path.exists(DRIVER) and os.access(DRIVER, os.X_OK)


def sample_molecules(name: str):
    """The molecules of a named sample and the (seed, atoms, noise) triples that rebuild them."""
    import numpy as np
    from stormm_b200 import synthetic
    workload, count, _, _ = SAMPLES[name]
    if workload == "batched_single_point":
        seed = synthetic.SEED_BASE + 1
        sizes = synthetic.batched_sizes(1024, seed=seed)
        seeds = [(synthetic._seed(seed, k), int(sizes[k]), 0.1) for k in range(count)]
        return [synthetic.make_molecule(s, n, noise=z) for (s, n, z) in seeds], seeds
    if workload == "minimization":
        seed = synthetic.SEED_BASE + 2
        sizes = np.random.default_rng(seed).integers(24, 97, size=4096)
        seeds = [(synthetic._seed(seed, k), int(sizes[k]), 0.3) for k in range(count)]
        return [synthetic.make_molecule(s, n, noise=z) for (s, n, z) in seeds], seeds
    seed = synthetic.SEED_BASE + 4
    sizes = np.random.default_rng(seed).integers(2000, 5001, size=256)
    return [synthetic.make_chain(synthetic._seed(seed, k), int(sizes[k]))
            for k in range(count)], None


def _sample_dir(name: str) -> str:
    return os.path.join(SAMPLE_ROOT, name)


def prepare_samples(names=None) -> None:
    """Write the named samples (all by default) as prmtop / inpcrd pairs with an index file."""
    from stormm_b200 import prmtop
    for name in (names or SAMPLES):
        d = _sample_dir(name)
        index = os.path.join(d, "index.txt")
        if os.path.exists(index):
            continue
        os.makedirs(d, exist_ok=True)
        mols, _ = sample_molecules(name)
        lines = []
        for k, m in enumerate(mols):
            top = os.path.join(d, f"m{k}.top")
            crd = os.path.join(d, f"m{k}.crd")
            prmtop.write_prmtop(m, top)
            prmtop.write_inpcrd(m, crd)
            lines.append(f"m{k}.top m{k}.crd\n")
        with open(index + ".tmp", "w") as f:
            f.writelines(lines)
        os.replace(index + ".tmp", index)


def _sample_files(name: str):
    """(prmtop, inpcrd) paths of a prepared sample, preparing it first if needed: in a child
    process, so that the process that times STORMM maps no library of the package under test."""
    d = _sample_dir(name)
    index = os.path.join(d, "index.txt")
    if not os.path.exists(index):
        root = os.path.dirname(HERE)
        subprocess.run([sys.executable, "-c",
                        f"import sys; sys.path.insert(0, {root!r}); import oracle.cpu_baseline as c; "
                        f"c.prepare_samples([{name!r}])"], check=True)
    with open(index) as f:
        return [tuple(os.path.join(d, p) for p in line.split()) for line in f if line.strip()]


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


def run_sample(name: str, seconds: float = 10.0, nproc: int | None = None):
    """Aggregate evaluations (or minimizations) per second of the CPU baseline on a named sample.
    Returns a dict with value, unit, cores, kind, count, seconds."""
    _, count, minimize_cycles, sd_cycles = SAMPLES[name]
    nproc = nproc or os.cpu_count() or 1
    nproc = max(1, min(nproc, count))
    what = "minimizations" if minimize_cycles > 0 else "evals"
    if reference_available():
        files = _sample_files(name)
        with tempfile.TemporaryDirectory() as tmp:
            lists = []
            for p in range(nproc):
                path = os.path.join(tmp, f"shard{p}.txt")
                with open(path, "w") as f:
                    for k in range(p, len(files), nproc):
                        f.write(f"{files[k][0]} {files[k][1]}\n")
                lists.append(path)
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
        _, seeds = sample_molecules(name)
        if seeds is None:
            raise RuntimeError("reference CPU build missing and the oracle port has no chains")
        ctx = mp.get_context("spawn")
        shards = [seeds[p::nproc] for p in range(nproc)]
        with ctx.Pool(nproc) as pool:
            res = pool.map(_port_worker, [(p, seconds, minimize_cycles, sd_cycles, shards[p])
                                          for p in range(nproc)])
        total = sum(r[0] for r in res)
        tmax = max(r[1] for r in res)
        kind = "port"
    return {"value": total / tmax,
            "unit": f"{'minimizations' if minimize_cycles else 'force-evals'}/s",
            "cores": nproc, "kind": kind, "count": total, "seconds": tmax, "molecules": count}
