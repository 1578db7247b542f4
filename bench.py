"""Benchmark of the batched implicit-solvent path on B200: single points and minimizations.

Headline workload (value): 1,024 distinct synthetic molecules with 16-256 atoms (uniform), OBC-II
GB (dielectric 80, no salt), Coulomb + Lennard-Jones with 1-2/1-3/1-4 exclusions and scaled 1-4
pairs, valence terms; FP32 arithmetic with int64 fixed-point forces (2^-23) and energies
(2^-26).  A step is one force + energy evaluation of every molecule: clearing the accumulators
and one fused launch.

Second workload (the "minimization" object): 4,096 molecules with 24-96 atoms, starting
coordinates perturbed by 0.3 A, 500 line-minimization cycles (50 steepest descent, then
conjugate gradient, no clash damping), each cycle a force evaluation and three energy-only
trial points; one step is one whole minimization of every molecule.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 the benchmark runs one process per GPU: under torchrun (RANK / WORLD_SIZE set) or,
without it, by spawning N ranks itself.  The ranks take disjoint shards of one seeded workload
of N x 1,024 (and N x 4,096) molecules, partitioned by pair count largest first
(stormm_b200.sharding.partition_lpt): weak scaling with no collective on the data path; the
only collectives are the barriers around timed regions and the max over ranks of the timing.
Rank 0 prints the details of every leg on one line and the summary on the last line.

Comparison points printed beside the numbers: STORMM's CPU build on the host cores
(cpu_baseline, oracle/cpu_baseline.py) and, where oracle/ref_gpu/Makefile has built it,
STORMM's own CUDA path on the same GPU and molecules (reference_gpu, oracle/gpu_reference.py).
"""
from __future__ import annotations

import argparse
import functools
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NSYS = 1024
WORKLOAD = "batched single point: 1024 molecules, 16-256 atoms, OBC-II GB, valence + Coulomb/LJ"
METRIC = "force-evals/s (batched single point, 1024 molecules of 16-256 atoms)"
# dram__bytes_read.sum + dram__bytes_write.sum of one kEvalFused launch on the 1,024-molecule
# single point, from the ncu capture summarized in profiles/ (the bench cannot profile itself)
KEVALFUSED_TRAFFIC_BYTES = 85.669376e6 + 81.111296e6
MIN_NSYS = 4096
MIN_CYCLES = 500
MIN_SD_CYCLES = 50
MIN_WORKLOAD = ("batched conformer minimization: 4096 molecules, 24-96 atoms, 0.3 A start noise, "
                "500 cycles (50 SD then CG), OBC-II GB")
LARGE_NSYS = 256
LARGE_WORKLOAD = ("large implicit-solvent systems: 256 polymer-like chains of 2000-5000 atoms "
                  "(seeded random walk, 1.5 A bonds, 2.5 A clash rejection), OBC-II GB, "
                  "force + energy, tiled path")
SERVED_RATES = (250.0, 1000.0, 4000.0)
SERVED_WINDOW_S = 1.0
SERVED_WORKLOAD = ("served minimization stream: Poisson arrivals, lognormal sizes (median 48 atoms, "
                   "sigma 0.6, clipped 12-512), 0.3 A start noise, each to RMS force <= 0.01 "
                   "kcal/mol/A or 2000 cycles")
TERMS = ["bond", "angle", "proper_dihedral", "improper_dihedral", "vdw", "vdw_14", "elec",
         "elec_14", "gb"]
ENERGY_BOUND = ("each term: |E - E_fp64| <= 1e-6 x max(|E_fp64|, 1 kcal/mol, root-sum-square of "
                "the term's contributions); forces: RMS relative error <= 5e-6")


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-minimization", action="store_true")
    ap.add_argument("--min-steps", type=int, default=2)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-errors", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--reference-gpu-full", action="store_true",
                    help="compare with STORMM's CUDA path on the whole workloads (slow set-up)")
    return ap.parse_args()


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device),
                                      f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        smax = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 4 + k and "Active" in s[4 + k] and "Not" not in s[4 + k]:
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------------------------------------
# Workloads: one seeded set of world x n molecules, an LPT shard per rank
# ------------------------------------------------------------------------------------------------
def _shard(sizes, world, rank):
    from stormm_b200 import sharding
    if world == 1:
        return np.arange(len(sizes))
    return sharding.partition_lpt(sizes, world)[rank]


@functools.lru_cache(maxsize=None)
def single_point_molecules(world, rank):
    from stormm_b200 import synthetic
    seed = synthetic.SEED_BASE + 1
    sizes = synthetic.batched_sizes(world * NSYS, seed=seed)
    idx = _shard(sizes, world, rank)
    return [synthetic.make_molecule(synthetic._seed(seed, int(k)), int(sizes[k]), noise=0.1,
                                    name=f"S{k}") for k in idx]


@functools.lru_cache(maxsize=None)
def minimization_molecules(world, rank):
    from stormm_b200 import synthetic
    seed = synthetic.SEED_BASE + 2
    sizes = np.random.default_rng(seed).integers(24, 97, size=world * MIN_NSYS)
    idx = _shard(sizes, world, rank)
    return [synthetic.make_molecule(synthetic._seed(seed, int(k)), int(sizes[k]), noise=0.3,
                                    name=f"N{k}") for k in idx]


def large_molecules(world, rank):
    from stormm_b200 import synthetic
    seed = synthetic.SEED_BASE + 4
    sizes = np.random.default_rng(seed).integers(2000, 5001, size=world * LARGE_NSYS)
    idx = _shard(sizes, world, rank)
    return [synthetic.make_chain(synthetic._seed(seed, int(k)), int(sizes[k]), name=f"C{k}")
            for k in idx]


# ------------------------------------------------------------------------------------------------
# Reference arm: STORMM's own CPU build on this host's cores
# ------------------------------------------------------------------------------------------------
def run_reference(args):
    """STORMM's own CPU code (oracle/_ref, built from the reference sources) on this host's
    cores over prebuilt Amber inputs of the workload's leading molecules."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    import oracle.cpu_baseline as cpub
    step_seconds = max(1.0, min(4.0, 60.0 / max(1, args.steps + args.warmup)))
    values = []
    info = None
    for s in range(args.warmup + args.steps):
        info = cpub.run_sample("single_point", step_seconds)
        if s >= args.warmup:
            values.append(info["value"])
    value = float(np.mean(values))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "force-evals/s",
        "n_gpus": max(world, args.gpus), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(NSYS / value * 1000.0), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded), the workload's first 256 molecules as the bounded sample",
        "config": {"workload": WORKLOAD, "molecules": NSYS, "atoms": "16-256", "gb": "OBC-II",
                   "sample_molecules": info["molecules"], "hardware": "host CPU cores"},
        "cpu_baseline": {"value": value, "unit": "force-evals/s", "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": f"{info['molecules']} molecules, {step_seconds:.1f} s per "
                                   f"step, one single-threaded FP64 process per core"},
        "e2e": {"value": value, "unit": "force-evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_minimization:
        m = cpub.run_sample("minimization", max(4.0, args.cpu_seconds))
        line["minimization"] = {"value": m["value"], "unit": "minimizations/s",
                                "workload": MIN_WORKLOAD, "cores": m["cores"], "kind": m["kind"],
                                "sample": f"{m['molecules']} molecules, {MIN_CYCLES} cycles each"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# Accuracy against the FP64 oracle (outside every timed region)
# ------------------------------------------------------------------------------------------------
def fp64_errors(mols, energies, forces, coords=None):
    """Largest per-term energy error relative to max(|E|, 1 kcal/mol), the largest ratio of error
    to the tests' bound (ENERGY_BOUND), and the largest force RMS relative error, over molecules
    evaluated by the FP64 oracle at the same coordinates."""
    import oracle
    rel = np.zeros(len(TERMS))
    ratio = np.zeros(len(TERMS))
    frel = 0.0
    fabs = 0.0
    for k, m in enumerate(mols):
        c = m.coords if coords is None else coords[k]
        osys = oracle.from_molecule(m)
        r = osys.evaluate(c)
        rss = osys.magnitudes(c, r["radii"])
        err = np.abs(np.asarray(energies[k]) - r["energies"])
        scale = np.maximum(np.abs(r["energies"]), 1.0)
        rel = np.maximum(rel, err / scale)
        ratio = np.maximum(ratio, err / (1e-6 * np.maximum(scale, rss)))
        f = np.asarray(forces[k])
        frel = max(frel, float(np.sqrt(((f - r["forces"]) ** 2).sum() /
                                       (r["forces"] ** 2).sum())))
        fabs = max(fabs, float(np.sqrt(((f - r["forces"]) ** 2).mean())))
    return {"molecules": len(mols), "bound": ENERGY_BOUND,
            "bound_ratio_max": float(ratio.max()),
            "energy_rel_max": {t: float(v) for t, v in zip(TERMS, rel)},
            "force_rms_rel_max": frel, "force_rms_abs_max_kcal_mol_A": fabs}


# ------------------------------------------------------------------------------------------------
# GPU legs
# ------------------------------------------------------------------------------------------------
def _event_pair():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    from stormm_b200 import sharding
    return sharding.max_over_ranks(x, device="cuda")


def _barrier(world: int):
    if world > 1:
        import torch
        torch.distributed.barrier()


E2E_BATCHES_IN_FLIGHT = 3


def _e2e_pipelined(args, world, mols, xyz, syn, local):
    """End-to-end force evaluations per second with E2E_BATCHES_IN_FLIGHT batches in flight,
    each with its own synthesis, stream and page-locked buffers (see the caller)."""
    import torch
    import stormm_b200 as sb
    depth = E2E_BATCHES_IN_FLIGHT
    others = [sb.Synthesis(mols, device=local) for _ in range(depth - 1)]
    syns = [syn] + others
    streams = [torch.cuda.Stream(device=local) for _ in range(depth)]
    done = [torch.cuda.Event() for _ in range(depth)]
    pin_in = [torch.from_numpy(xyz.copy()).pin_memory().numpy() for _ in range(depth)]
    pin_f = [torch.zeros(xyz.size, dtype=torch.float64).pin_memory().numpy()
             for _ in range(depth)]
    pin_e = [torch.zeros(len(mols) * sb.NRG_STRIDE, dtype=torch.float64).pin_memory().numpy()
             for _ in range(depth)]
    pending = [False] * depth
    sums = []

    def take(b):
        done[b].synchronize()
        if pending[b]:
            sums.append(float(pin_e[b].sum()))
            pending[b] = False

    def step(k):
        b = k % depth
        take(b)
        h = streams[b].cuda_stream
        syns[b].set_coordinates(pin_in[b], stream=h)
        syns[b].initialize(sb.INIT_FORCES | sb.INIT_ENERGIES, stream=h)
        syns[b].evaluate(stream=h)
        syns[b].download_async(pin_f[b], pin_e[b], stream=h)
        done[b].record(streams[b])
        pending[b] = True

    for k in range(2 * depth):
        step(k)
    for b in range(depth):
        take(b)
    sums.clear()
    torch.cuda.synchronize()
    _barrier(world)
    t0 = time.perf_counter()
    for k in range(args.steps):
        step(k)
    for b in range(depth):
        take(b)
    torch.cuda.synchronize()
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
    for o in others:
        o.close()
    assert len(sums) == args.steps
    return world * NSYS * args.steps / e2e_s, sums


def bench_single_point(args, world, rank, local, flush):
    import torch
    import stormm_b200 as sb
    from stormm_b200 import roofline

    mols = single_point_molecules(world, rank)
    natoms = np.array([m.natom for m in mols])
    syn = sb.Synthesis(mols, device=local)
    xyz = np.concatenate([m.coords for m in mols])
    syn.set_coordinates(xyz)
    info = syn.launch_info()

    def step():
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    assert syn.status() == 0

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kbeg = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    _barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record()
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        kbeg[k].record()
        syn.evaluate()
        ends[k].record()
    torch.cuda.synchronize()
    _barrier(world)
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    kern_ms = np.array([s.elapsed_time(e) for s, e in zip(kbeg, ends)])
    total_ms = _max_over_ranks(float(step_ms.sum()), world)
    value = world * NSYS * args.steps / (total_ms / 1000.0)
    errors = None
    if rank == 0 and not args.no_errors:
        errors = fp64_errors(mols, syn.energy_terms(), syn.split(syn.forces()))

    # end to end through the C ABI with host buffers: upload coordinates, evaluate, read back
    # forces and energies every step (pinned host buffers, allocated once and reused, as a
    # serving loop would)
    pinned_xyz = torch.from_numpy(xyz.copy()).pin_memory().numpy()
    pinned_f = torch.zeros(xyz.size, dtype=torch.float64).pin_memory().numpy()
    pinned_e = torch.zeros(len(mols) * sb.NRG_STRIDE, dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        syn.set_coordinates(pinned_xyz)
        step()
        syn.forces(out=pinned_f)
        syn.energies(out=pinned_e)
    torch.cuda.synchronize()
    _barrier(world)
    t0 = time.perf_counter()
    lat = []
    for _ in range(args.steps):
        ts = time.perf_counter()
        syn.set_coordinates(pinned_xyz)
        step()
        f = syn.forces(out=pinned_f)
        e = syn.energies(out=pinned_e)
        lat.append(time.perf_counter() - ts)
    torch.cuda.synchronize()
    e2e_sync_s = _max_over_ranks(time.perf_counter() - t0, world)
    e2e_sync_value = world * NSYS * args.steps / e2e_sync_s

    # the same steps as a serving loop runs them: several batches in flight on their own
    # streams, each step's upload, evaluation and asynchronous read-back enqueued on its batch's
    # stream, so one batch's transfers overlap the others' evaluations; the host takes each
    # step's results (the sum of its energies) once its stream has finished them
    e2e_value, e2e_sums = _e2e_pipelined(args, world, mols, xyz, syn, local)

    # per-system drop-in: one launch per molecule (same kernel, one molecule each)
    per_sys = None
    if rank == 0:
        n = len(mols)
        syn.initialize()
        syn.evaluate_range(0, n)
        torch.cuda.synchronize()
        ev0, ev1 = _event_pair()
        reps = 3
        ev0.record()
        for _ in range(reps):
            syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
            syn.evaluate_range(0, n)
        ev1.record()
        torch.cuda.synchronize()
        per_sys = n * reps / (ev0.elapsed_time(ev1) / 1000.0)
    syn.close()

    flops = roofline.flops_per_evaluation(natoms, force=True)
    return {
        "value": value, "total_ms": total_ms, "step_ms": step_ms, "natoms": natoms,
        "info": info, "per_sys": per_sys, "e2e_value": e2e_value, "lat": lat,
        "e2e_sync_value": e2e_sync_value, "e2e_sums": e2e_sums,
        "h2d": int(xyz.size * 8), "d2h": int(f.size * 8 + e.size * 8),
        "flops": flops, "kern_avg_s": float(kern_ms.mean()) / 1000.0, "errors": errors,
    }


def bench_minimization(args, world, rank, local, flush):
    import torch
    import oracle
    import stormm_b200 as sb

    mols = minimization_molecules(world, rank)
    syn = sb.Synthesis(mols, device=local)
    xyz = np.concatenate([m.coords for m in mols])
    ctl = dict(total_cycles=MIN_CYCLES, sd_cycles=MIN_SD_CYCLES, kernel=sb.MIN_GRAPH)
    syn.set_coordinates(xyz)
    # untimed: the graph minimizer's evaluations use the evaluation packing
    tuned = syn.autotune(sb.TUNE_EVALUATE)
    for _ in range(3):
        syn.set_coordinates(xyz)
        syn.minimize(total_cycles=5, sd_cycles=2, kernel=sb.MIN_GRAPH)
    torch.cuda.synchronize()
    assert syn.status() == 0
    times = []
    _barrier(world)
    for _ in range(args.min_steps):
        syn.set_coordinates(xyz)
        flush.zero_()
        ev0, ev1 = _event_pair()
        ev0.record()
        syn.minimize(**ctl)
        ev1.record()
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
    _barrier(world)
    total_ms = _max_over_ranks(float(np.sum(times)), world)
    value = world * MIN_NSYS * args.min_steps / (total_ms / 1000.0)
    e_final_terms = syn.energy_terms()
    e_final = e_final_terms.sum(axis=1)
    errors = None
    if rank == 0 and not args.no_errors:
        # accuracy at the minimized coordinates: an untimed force + energy evaluation there
        # against the oracle, and the trajectory of the first 8 molecules against the oracle's
        # restatement of STORMM's GPU line search over all 500 cycles
        final_xyz = syn.split(syn.coordinates())
        syn.initialize()
        syn.evaluate()
        errors = fp64_errors(mols, syn.energy_terms(), syn.split(syn.forces()), final_xyz)
        errors["note"] = ("at minimized coordinates the forces approach zero, so their relative "
                          "error is large by construction; the absolute RMS error is the measure")
        traj = []
        for k in range(8):
            _, hist = oracle.from_molecule(mols[k]).minimize(mols[k].coords, MIN_CYCLES,
                                                             MIN_SD_CYCLES)
            drop = hist[0] - hist[-1]
            traj.append(abs(e_final[k] - hist[-1]) / max(abs(drop), 1e-12))
        errors["final_energy_vs_oracle_trajectory"] = {
            "molecules": 8, "max_abs_diff_over_energy_drop": float(np.max(traj)),
            "median": float(np.median(traj))}
    # end to end: pinned host coordinates in, minimize, coordinates and energies out
    pinned_xyz = torch.from_numpy(xyz.copy()).pin_memory().numpy()
    pinned_c = torch.zeros(xyz.size, dtype=torch.float64).pin_memory().numpy()
    pinned_e = torch.zeros(len(mols) * sb.NRG_STRIDE, dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    _barrier(world)
    t0 = time.perf_counter()
    syn.set_coordinates(pinned_xyz)
    syn.minimize(**ctl)
    c = syn.coordinates(out=pinned_c)
    e = syn.energies(out=pinned_e)
    e2e_s = _max_over_ranks(time.perf_counter() - t0, world)
    # per-system drop-in: one launch sequence per molecule for the first 16 molecules
    per_sys = None
    e_start = None
    if rank == 0:
        syn.set_coordinates(xyz)
        ev0, ev1 = _event_pair()
        ev0.record()
        syn.minimize_range(0, 16, **ctl)
        ev1.record()
        torch.cuda.synchronize()
        per_sys = 16 / (ev0.elapsed_time(ev1) / 1000.0)
        syn.set_coordinates(xyz)
        syn.initialize()
        syn.evaluate(force=False, energy=True)
        e_start = syn.energy_terms().sum(axis=1)
    # the persistent-kernel minimizer on the same workload, one run, for comparison
    syn.set_coordinates(xyz)
    syn.autotune(sb.TUNE_MINIMIZE)
    syn.set_coordinates(xyz)
    ev0, ev1 = _event_pair()
    ev0.record()
    syn.minimize(total_cycles=MIN_CYCLES, sd_cycles=MIN_SD_CYCLES, kernel=sb.MIN_PERSISTENT)
    ev1.record()
    torch.cuda.synchronize()
    persistent = len(mols) / (ev0.elapsed_time(ev1) / 1000.0)
    assert syn.status() == 0
    syn.close()
    fp64_mode = None
    if rank == 0:
        fp64_mode = _minimization_fp64(mols[:256], e_final[:256], local)
    evals = MIN_NSYS * (4 * MIN_CYCLES + 1)
    return {
        "value": value, "unit": "minimizations/s", "workload": MIN_WORKLOAD,
        "molecules_per_gpu": MIN_NSYS, "cycles": MIN_CYCLES, "sd_cycles": MIN_SD_CYCLES,
        "clash_cycles": 0, "steps": args.min_steps, "ms_per_step": total_ms / args.min_steps,
        "p50_ms": float(np.percentile(times, 50)), "p99_ms": float(np.percentile(times, 99)),
        "evals_per_s": world * evals * args.min_steps / (total_ms / 1000.0),
        "evals_per_minimization": 4 * MIN_CYCLES + 1,
        "per_system_dropin": {"value": per_sys, "unit": "minimizations/s",
                              "sample": "first 16 molecules, one launch sequence each"},
        "batched_speedup": (value / world / per_sys) if per_sys else None,
        "e2e": {"value": world * MIN_NSYS / e2e_s, "unit": "minimizations/s",
                "h2d_bytes_per_step": int(xyz.size * 8),
                "d2h_bytes_per_step": int(c.size * 8 + e.size * 8)},
        "mean_energy_drop": (float(np.mean(e_start - e_final)) if e_start is not None else None),
        "mean_final_energy": float(np.mean(e_final)),
        "kernel": "graph (one CUDA graph per cycle: 4 batched evaluations + 4 line-search kernels)",
        "persistent_kernel_value": persistent,
        "fp64_mode": fp64_mode,
        "gpu_launches_per_step": 1 + 8 * MIN_CYCLES + 2,
        "unit_packing": {"atoms_per_unit": tuned[0], "tiles_per_unit": tuned[1],
                         "chosen_by": "sb_autotune of the evaluation"},
        "l2": "flushed (256 MB write) before every timed step",
        "errors": errors,
    }


def _minimization_fp64(mols, e_fp32_final, local):
    """The FP64 mode (PrecisionModel::DOUBLE) on the first 256 molecules: one timed run after a
    short warm-up, and the FP32 path's final energies against its own."""
    import torch
    import stormm_b200 as sb
    x64 = np.concatenate([m.coords for m in mols])
    s64 = sb.Synthesis(mols, device=local, precision=sb.PRECISION_DOUBLE)
    s64.set_coordinates(x64)
    s64.minimize(total_cycles=5, sd_cycles=2, kernel=sb.MIN_GRAPH)
    s64.set_coordinates(x64)
    torch.cuda.synchronize()
    ev0, ev1 = _event_pair()
    ev0.record()
    s64.minimize(total_cycles=MIN_CYCLES, sd_cycles=MIN_SD_CYCLES, kernel=sb.MIN_GRAPH)
    ev1.record()
    torch.cuda.synchronize()
    value = len(mols) / (ev0.elapsed_time(ev1) / 1000.0)
    e64 = s64.energy_terms().sum(axis=1)
    assert s64.status() == 0
    s64.close()
    return {"value": value, "unit": "minimizations/s", "molecules": len(mols),
            "cycles": MIN_CYCLES,
            "fp32_final_energy_rel_vs_fp64_median": float(np.median(
                np.abs(e_fp32_final - e64) / np.maximum(np.abs(e64), 1.0))),
            "note": "graph minimizer over the FP64 evaluations, conjugate direction in FP64"}


def bench_large(args, world, rank, local, flush):
    """256 chains of 2,000-5,000 atoms through the tiled path."""
    import torch
    import stormm_b200 as sb
    from stormm_b200 import roofline
    mols = large_molecules(world, rank)
    natoms = np.array([m.natom for m in mols])
    syn = sb.Synthesis(mols, device=local)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    for _ in range(3):
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate()
    torch.cuda.synchronize()
    assert syn.status() == 0
    times = []
    _barrier(world)
    for _ in range(5):
        flush.zero_()
        ev0, ev1 = _event_pair()
        ev0.record()
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate()
        ev1.record()
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
    _barrier(world)
    total_ms = _max_over_ranks(float(np.sum(times)), world)
    value = world * LARGE_NSYS * len(times) / (total_ms / 1000.0)
    fp64 = None
    per_sys = None
    if rank == 0:
        fp64 = _large_fp64(mols, local, syn.forces(), syn.energy_terms(), flush)
        ev0, ev1 = _event_pair()
        ev0.record()
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate_range(0, 16)
        ev1.record()
        torch.cuda.synchronize()
        per_sys = 16 / (ev0.elapsed_time(ev1) / 1000.0)
    syn.close()
    flops = roofline.flops_per_evaluation(natoms, force=True)
    achieved = flops / (float(np.mean(times)) / 1000.0) / 1.0e12
    peak = roofline.fp32_peak_tflops(1965.0)
    return {"workload": LARGE_WORKLOAD, "value": value, "unit": "force-evals/s",
            "molecules_per_gpu": LARGE_NSYS, "atoms_total_per_gpu": int(natoms.sum()),
            "pairs_per_pass": roofline.pair_count(natoms), "steps": len(times),
            "ms_per_step": total_ms / len(times),
            "p50_ms": float(np.percentile(times, 50)), "p99_ms": float(np.percentile(times, 99)),
            "per_system_dropin": {"value": per_sys, "unit": "force-evals/s",
                                  "sample": "first 16 chains, one launch sequence each"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "flops_per_step": flops},
            "l2": "flushed (256 MB write) before every timed step",
            "fp64_gpu_mode": fp64}


def _large_fp64(mols, local, f32, e32, flush, steps=3):
    """The same chains in the FP64-arithmetic mode: its throughput on one GPU, and how far the
    FP32 path's forces and energies lie from it."""
    import torch
    import stormm_b200 as sb
    syn = sb.Synthesis(mols, device=local, precision=sb.PRECISION_DOUBLE)
    syn.set_coordinates(np.concatenate([m.coords for m in mols]))
    syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
    syn.evaluate()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        ev0, ev1 = _event_pair()
        ev0.record()
        syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
        syn.evaluate()
        ev1.record()
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
    assert syn.status() == 0
    f64 = syn.forces()
    e64 = syn.energy_terms()
    syn.close()
    frel = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))
    rel = np.max(np.abs(e32 - e64) / np.maximum(np.abs(e64), 1.0), axis=0)
    return {"value": len(mols) * steps / (float(np.sum(times)) / 1000.0),
            "unit": "force-evals/s", "steps": steps, "ms_per_step": float(np.mean(times)),
            "n_gpus": 1, "fp32_force_rms_rel_vs_fp64": frel,
            "fp32_energy_rel_vs_fp64_max": {t: float(v) for t, v in zip(TERMS, rel)}}


def bench_served(local):
    """Poisson request streams at several rates through the continuous-batching server."""
    import stormm_b200 as sb
    from stormm_b200 import synthetic
    mols = synthetic.workload_served(1600)
    srv = sb.Server(options=sb.default_options(device=local))
    prepared = [srv.prepare(m) for m in mols]
    srv.close()
    sweeps = []
    for rate in SERVED_RATES:
        srv = sb.Server(options=sb.default_options(device=local), cycles_per_launch=50)
        rng = np.random.default_rng(int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * SERVED_WINDOW_S * 2) + 8))
        arrivals = arrivals[arrivals < SERVED_WINDOW_S]
        start = time.perf_counter()
        for k, ta in enumerate(arrivals):
            while time.perf_counter() - start < ta:
                pass
            srv.submit(mols[k % len(mols)], prepared=prepared[k % len(mols)])
        drained = srv.drain(600.0)
        res = [r for r, _ in srv.poll(max_results=len(arrivals) + 16, coordinates=False)]
        moved = srv.stats()["migrated"]
        srv.close()
        lat = np.array([r["finish_time"] - r["submit_time"] for r in res])
        wait = np.array([r["admit_time"] - r["submit_time"] for r in res])
        first = min(r["submit_time"] for r in res)
        last = max(r["finish_time"] for r in res)
        sweeps.append({
            "offered_per_s": rate, "requests": len(arrivals), "completed": len(res),
            "drained": bool(drained),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "admission_wait_p50_ms": float(np.percentile(wait, 50) * 1e3),
            "throughput_per_s": len(res) / (last - first),
            "mean_cycles": float(np.mean([r["cycles"] for r in res])),
            "converged_fraction": float(np.mean([r["converged"] for r in res])),
            "migrated": int(moved),
        })
    # A mixed stream: every other request a force + energy evaluation, the rest minimizations
    rate = 1000.0
    srv = sb.Server(options=sb.default_options(device=local), cycles_per_launch=50)
    rng = np.random.default_rng(4242)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * SERVED_WINDOW_S * 2) + 8))
    arrivals = arrivals[arrivals < SERVED_WINDOW_S]
    start = time.perf_counter()
    for k, ta in enumerate(arrivals):
        while time.perf_counter() - start < ta:
            pass
        srv.submit(mols[k % len(mols)], prepared=prepared[k % len(mols)], evaluate=(k % 2 == 1))
    drained = srv.drain(600.0)
    res = [r for r, _ in srv.poll(max_results=len(arrivals) + 16, coordinates=False)]
    srv.close()
    mixed = {"offered_per_s": rate, "evaluation_share": 0.5, "requests": len(arrivals),
             "completed": len(res), "drained": bool(drained)}
    for kind in ("evaluate", "minimize"):
        lat = np.array([r["finish_time"] - r["submit_time"] for r in res if r["kind"] == kind])
        if lat.size:
            mixed[kind] = {"completed": int(lat.size),
                           "p50_ms": float(np.percentile(lat, 50) * 1e3),
                           "p99_ms": float(np.percentile(lat, 99) * 1e3)}
    return {"workload": SERVED_WORKLOAD, "unit": "requests/s, latency ms (submit to result)",
            "arrival_window_s": SERVED_WINDOW_S, "cycles_per_launch": 50,
            "throughput_note": "completions over first submit to last result, drain tail included",
            "sweep": sweeps, "mixed_with_evaluations": mixed}


def _cpu_leg(name, seconds):
    """STORMM's CPU build on this host's cores over the named sample (oracle.cpu_baseline)."""
    import oracle.cpu_baseline as cpub
    try:
        r = cpub.run_sample(name, seconds)
        return {"value": r["value"], "unit": r["unit"], "cores": r["cores"], "kind": r["kind"],
                "sample": f"the workload's first {r['molecules']} molecules, {seconds:.0f} s, "
                          f"one single-threaded FP64 process per core"}
    except Exception as exc:  # reported, not fatal
        return {"value": None, "unit": None, "cores": 0, "kind": "unavailable",
                "sample": str(exc)[:200]}


REF_GPU_SP_SAMPLE = 256       # molecules of each workload the reference CUDA leg compares on
REF_GPU_MIN_SAMPLE = 512


def _this_path_on(mols, local, evals, minimize_cycles=0, sd_cycles=0):
    """This path on the comparison sample, timed the way the reference CUDA leg times STORMM:
    back-to-back force + energy evaluations (CUDA events, no L2 flush), or the wall time of one
    minimization call after an untimed one with the same controls."""
    import torch
    import stormm_b200 as sb
    syn = sb.Synthesis(mols, device=local)
    xyz = np.concatenate([m.coords for m in mols])
    syn.set_coordinates(xyz)
    try:
        if minimize_cycles == 0:
            for _ in range(3):
                syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
                syn.evaluate()
            torch.cuda.synchronize()
            e0, e1 = _event_pair()
            e0.record()
            for _ in range(evals):
                syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
                syn.evaluate()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            return {"value": len(mols) * evals / (ms / 1000.0), "ms_per_eval": ms / evals}
        ctl = dict(total_cycles=minimize_cycles, sd_cycles=sd_cycles, kernel=sb.MIN_GRAPH)
        syn.minimize(**ctl)
        syn.set_coordinates(xyz)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        syn.minimize(**ctl)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1000.0
        return {"value": len(mols) / (ms / 1000.0), "ms": ms}
    finally:
        syn.close()


def _reference_gpu_leg(args, local):
    """STORMM's own CUDA path (oracle/_ref_gpu, built from the reference sources by
    oracle/ref_gpu/Makefile) against this path on the same GPU and the same molecules:
    launchNonbonded + launchValence against the fused evaluation, launchMinimization against
    the graph minimizer, STORMM's in a subprocess that maps only STORMM's library and CUDA's.
    STORMM's host set-up of a synthesis grows steeply with the number of distinct topologies
    (about 4 minutes for the 1,024 molecules of the single point, 13 for the 4,096 of the
    minimization batch, measured on the B200 host), so by default both run on the workloads'
    leading molecules (REF_GPU_SP_SAMPLE, REF_GPU_MIN_SAMPLE) and --reference-gpu-full runs the
    whole workloads.  A failure is reported, not fatal."""
    from oracle import gpu_reference as gref
    if not gref.available():
        return {"available": False, "why": "reference CUDA build absent (oracle/ref_gpu/Makefile)"}
    out = {"available": True,
           "build": "STORMM's sources with its CUDA path, nvcc -O3 --use_fast_math sm_100",
           "precision": "STORMM PrecisionModel::SINGLE (FP32, split fixed-point accumulation)"}
    full = args.reference_gpu_full
    evals = max(20, args.steps)
    try:
        mols = single_point_molecules(1, 0)
        mols = mols if full else mols[:REF_GPU_SP_SAMPLE]
        lst = gref.write_inputs(f"single_point_{len(mols)}", mols)
        r = gref.time_evaluations(lst, evals)
        ours = _this_path_on(mols, local, evals)
        out["single_point"] = {
            "value": r["value"], "unit": "force-evals/s", "ms_per_eval": r["ms_per_eval"],
            "this_path_value": ours["value"], "this_path_ms_per_eval": ours["ms_per_eval"],
            "ratio_this_path": ours["value"] / r["value"],
            "molecules": len(mols), "atoms": r["atoms"], "evals": r["evals"],
            "timing": "both: CUDA events over back-to-back force + energy evaluations (clear the "
                      "accumulators, evaluate), L2 not flushed"}
    except Exception as exc:  # reported, not fatal
        out["single_point"] = {"error": str(exc)[:300]}
    if not args.no_minimization:
        try:
            mols = minimization_molecules(1, 0)
            mols = mols if full else mols[:REF_GPU_MIN_SAMPLE]
            lst = gref.write_inputs(f"minimization_{len(mols)}", mols)
            with tempfile.TemporaryDirectory() as tmp:
                r = gref.minimize(lst, os.path.join(tmp, "min.bin"), MIN_CYCLES, MIN_SD_CYCLES,
                                  ntpr=MIN_CYCLES)
            ours = _this_path_on(mols, local, 0, MIN_CYCLES, MIN_SD_CYCLES)
            out["minimization"] = {
                "value": r["value"], "unit": "minimizations/s", "ms": r["ms"],
                "this_path_value": ours["value"], "this_path_ms": ours["ms"],
                "ratio_this_path": ours["value"] / r["value"],
                "molecules": r["systems"], "cycles": MIN_CYCLES, "sd_cycles": MIN_SD_CYCLES,
                "timing": "wall time of one minimization call: STORMM's launchMinimization (its "
                          "launch set-up included), this path's graph minimizer (its cycle graph "
                          "captured by an untimed call)",
                "mean_final_energy": float(np.mean(r["final_terms"].sum(axis=1)))}
        except Exception as exc:  # reported, not fatal
            out["minimization"] = {"error": str(exc)[:300]}
    return out


def main_rank(args):
    world, rank, local = _dist()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from stormm_b200 import roofline

    # L2 flush buffer (> 126 MB L2), written between timed steps outside the timed events
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    with ClockSampler(local) as clocks:
        sp = bench_single_point(args, world, rank, local, flush)
        mn = None if args.no_minimization else bench_minimization(args, world, rank, local, flush)
        served = None if (args.no_served or rank != 0) else bench_served(local)
        large = None if args.no_large else bench_large(args, world, rank, local, flush)
    csum = clocks.summary()

    achieved = sp["flops"] / sp["kern_avg_s"] / 1.0e12
    peak = roofline.fp32_peak_tflops(1965.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = _cpu_leg("single_point", args.cpu_seconds)
        if mn is not None:
            mn["cpu_baseline"] = _cpu_leg("minimization", args.cpu_seconds)
        if large is not None:
            large["cpu_baseline"] = _cpu_leg("large", args.cpu_seconds)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = _reference_gpu_leg(args, local)

    if rank == 0:
        info = sp["info"]
        natoms = sp["natoms"]
        detail = {"detail": "bench legs in full (the summary line follows)",
                  "minimization": mn, "served": served, "large": large,
                  "reference_gpu": ref_gpu}
        print(json.dumps(detail, default=float), flush=True)
        line = {
            "metric": METRIC, "value": sp["value"], "unit": "force-evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sp["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (int64 fixed-point accumulation)",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOAD, "molecules_per_gpu": NSYS,
                       "atoms_per_gpu_rank0": int(natoms.sum()),
                       "pairs_per_pass_rank0": roofline.pair_count(natoms), "gb": "OBC-II",
                       "parallelism": (f"{world} ranks, LPT shards of one {world * NSYS}-molecule "
                                       f"workload" if world > 1 else "one GPU"),
                       "l2": "flushed (256 MB write) before every timed step",
                       "work_units": info["work_units"], "threads_per_block": info["threads"]},
            "p50_ms": float(np.percentile(sp["step_ms"], 50)),
            "p99_ms": float(np.percentile(sp["step_ms"], 99)),
            "per_system_dropin": {"value": sp["per_sys"], "unit": "force-evals/s",
                                  "batched_speedup": (sp["value"] / world / sp["per_sys"])
                                  if sp["per_sys"] else None},
            "e2e": {"value": sp["e2e_value"], "unit": "force-evals/s",
                    "h2d_bytes_per_step": sp["h2d"], "d2h_bytes_per_step": sp["d2h"],
                    "mode": f"{E2E_BATCHES_IN_FLIGHT} batches in flight on their own streams "
                            "(sb_download_results_async)",
                    "one_batch_at_a_time": sp["e2e_sync_value"],
                    "p50_ms": float(np.percentile(sp["lat"], 50)) * 1000.0,
                    "p99_ms": float(np.percentile(sp["lat"], 99)) * 1000.0},
            "gpu_launches": args.steps * (1 if info["work_units"] else 0),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": KEVALFUSED_TRAFFIC_BYTES,
                         "traffic_unit": "DRAM bytes read + written per launch",
                         "traffic_source": "ncu capture of this launch shape "
                                           "(profiles/kEvalFused_single_point_1024_molecules.md):"
                                           " 35 MB of inputs, the rest the pair-derivative store",
                         "kernel": "kEvalFused", "flops_per_launch": sp["flops"],
                         "kernel_ms": sp["kern_avg_s"] * 1000.0,
                         "peak_source": "nominal FP32 FMA pipe: 148 SM x 128 lanes x 2 x "
                                        "1965 MHz (no measured FP32 figure on this pool)"},
            "errors_vs_fp64": sp["errors"],
            "clocks": csum,
            "cpu_baseline": cpu,
        }
        if mn is not None:
            line["minimization"] = {
                "value": mn["value"], "unit": "minimizations/s", "workload": MIN_WORKLOAD,
                "evals_per_s": mn["evals_per_s"],
                "per_system_dropin": mn["per_system_dropin"]["value"],
                "batched_speedup": mn["batched_speedup"],
                "errors_vs_fp64": mn["errors"],
                "cpu_baseline": (mn.get("cpu_baseline") or {}).get("value")}
        if ref_gpu is not None and ref_gpu.get("available"):
            line["reference_gpu"] = {
                k: {f: v.get(f) for f in ("value", "this_path_value", "ratio_this_path",
                                          "molecules", "error") if f in v}
                for k, v in ref_gpu.items() if isinstance(v, dict)}
        print(json.dumps(line, default=float), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _rank_main(args):
    if args.impl == "reference":
        run_reference(args)
    else:
        main_rank(args)


def main():
    args = _args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU without torchrun
        from stormm_b200 import sharding
        sharding.spawn_ranks(_rank_main, args.gpus, args)
        return
    _rank_main(args)


if __name__ == "__main__":
    main()
