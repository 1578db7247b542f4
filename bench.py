"""Benchmark of the batched implicit-solvent single point (force + energy) on B200.

Workload: 1,024 distinct synthetic molecules with 16-256 atoms (uniform), OBC-II GB (dielectric
80, no salt), Coulomb + Lennard-Jones with 1-2/1-3/1-4 exclusions and scaled 1-4 pairs, valence
terms; FP32 arithmetic with int64 fixed-point forces (2^-23) and energies (2^-26).  A step is one
force + energy evaluation of every molecule: clearing the accumulators and one fused launch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun, one process per GPU; each rank evaluates its own 1,024 molecules
(weak scaling, no collective on the data path; the only collective is the max-over-ranks of the
timing).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NSYS = 1024
WORKLOAD = "batched single point: 1024 molecules, 16-256 atoms, OBC-II GB, valence + Coulomb/LJ"
METRIC = "force-evals/s (batched single point, 1024 molecules of 16-256 atoms)"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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


def _workload(rank: int):
    from stormm_b200 import synthetic
    return synthetic.workload_batched_single_point(NSYS, seed=synthetic.SEED_BASE + 1 + 1000 * rank)


def run_reference(args):
    """Reference arm: STORMM's own CPU evaluator on this host's cores, same metric/config."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    import oracle.cpu_baseline as cpub
    from stormm_b200 import synthetic
    sizes = synthetic.batched_sizes(NSYS)
    sample_n = 256
    mols = [synthetic.make_molecule(synthetic._seed(synthetic.SEED_BASE + 1, k), int(sizes[k]))
            for k in range(sample_n)]
    seeds = [(synthetic._seed(synthetic.SEED_BASE + 1, k), int(sizes[k]), 0.1)
             for k in range(sample_n)]
    step_seconds = max(1.0, min(4.0, 60.0 / max(1, args.steps + args.warmup)))
    values = []
    info = None
    for s in range(args.warmup + args.steps):
        info = cpub.run(mols, seconds=step_seconds, molecule_seeds=seeds)
        if s >= args.warmup:
            values.append(info["value"])
    value = float(np.mean(values))
    ms = float(NSYS / value * 1000.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "force-evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded), first 256 molecules of the workload as the bounded sample",
        "config": {"workload": WORKLOAD, "molecules": NSYS, "atoms": "16-256",
                   "gb": "OBC-II", "sample_molecules": sample_n},
        "cpu_baseline": {"value": value, "unit": "force-evals/s", "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": f"{sample_n} molecules, {step_seconds:.1f} s per step, "
                                   f"one single-threaded FP64 process per core"},
        "e2e": {"value": value, "unit": "force-evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
        return
    world, rank, local = _dist()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import stormm_b200 as sb
    from stormm_b200 import roofline

    mols = _workload(rank)
    natoms = np.array([m.natom for m in mols])
    syn = sb.Synthesis(mols, device=local)
    xyz = np.concatenate([m.coords for m in mols])
    syn.set_coordinates(xyz)
    info = syn.launch_info()

    # L2 flush buffer (> 126 MB L2), written between timed steps outside the timed events
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

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
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
            kbeg[k].record()
            syn.evaluate()
            ends[k].record()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
        kern_ms = np.array([s.elapsed_time(e) for s, e in zip(kbeg, ends)])
    total_ms = float(step_ms.sum())
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * NSYS * args.steps / (total_ms / 1000.0)

    # end to end through the C ABI with host buffers: upload coordinates, evaluate, read back
    # forces and energies every step
    pinned_xyz = torch.from_numpy(xyz.copy()).pin_memory().numpy()
    for _ in range(2):
        syn.set_coordinates(pinned_xyz)
        step()
        syn.forces()
        syn.energies()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    lat = []
    for _ in range(args.steps):
        ts = time.perf_counter()
        syn.set_coordinates(pinned_xyz)
        step()
        f = syn.forces()
        e = syn.energies()
        lat.append(time.perf_counter() - ts)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * NSYS * args.steps / e2e_s
    h2d = int(xyz.size * 8)
    d2h = int(f.size * 8 + e.size * 8)

    # per-system drop-in: one launch sequence per molecule (same kernels, one molecule each)
    per_sys = None
    if rank == 0:
        syn.initialize()
        syn.evaluate_range(0, NSYS)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        ev0.record()
        for _ in range(reps):
            syn.initialize(sb.INIT_FORCES | sb.INIT_ENERGIES)
            syn.evaluate_range(0, NSYS)
        ev1.record()
        torch.cuda.synchronize()
        per_sys = NSYS * reps / (ev0.elapsed_time(ev1) / 1000.0)

    flops = roofline.flops_per_evaluation(natoms, force=True)
    kern_avg_s = float(kern_ms.mean()) / 1000.0
    achieved = flops / kern_avg_s / 1.0e12
    peak = roofline.fp32_peak_tflops(1965.0)
    csum = clocks.summary()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle.cpu_baseline as cpub
            from stormm_b200 import synthetic
            sizes = synthetic.batched_sizes(NSYS)
            sample_n = 256
            sample = mols[:sample_n]
            seeds = [(synthetic._seed(synthetic.SEED_BASE + 1, k), int(sizes[k]), 0.1)
                     for k in range(sample_n)]
            r = cpub.run(sample, seconds=args.cpu_seconds, molecule_seeds=seeds)
            cpu = {"value": r["value"], "unit": "force-evals/s", "cores": r["cores"],
                   "kind": r["kind"],
                   "sample": f"first {sample_n} molecules of the workload, "
                             f"{args.cpu_seconds:.0f} s, one FP64 process per core"}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": "force-evals/s", "cores": 0, "kind": "unavailable",
                   "sample": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "force-evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (int64 fixed-point accumulation)",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOAD, "molecules_per_gpu": NSYS,
                       "atoms_total_per_gpu": int(natoms.sum()),
                       "pairs_per_pass": roofline.pair_count(natoms), "gb": "OBC-II",
                       "dielectric": 80.0, "parallelism": f"weak x{world} (independent shards)",
                       "l2": "flushed (256 MB write) before every timed step",
                       "work_units": info["work_units"], "threads_per_block": info["threads"]},
            "p50_ms": float(np.percentile(step_ms, 50)),
            "p99_ms": float(np.percentile(step_ms, 99)),
            "per_system_dropin": {"value": per_sys, "unit": "force-evals/s",
                                  "launches_per_step": NSYS,
                                  "batched_speedup": (value / world / per_sys) if per_sys else None},
            "e2e": {"value": e2e_value, "unit": "force-evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "p50_ms": float(np.percentile(lat, 50)) * 1000.0,
                    "p99_ms": float(np.percentile(lat, 99)) * 1000.0},
            "gpu_launches": args.steps * (1 if info["work_units"] else 0),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "kernel": "kEvalFused", "flops_per_launch": flops,
                         "kernel_ms": kern_avg_s * 1000.0,
                         "peak_source": "nominal FP32 FMA pipe: 148 SM x 128 lanes x 2 x 1965 MHz"},
            "clocks": csum,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    syn.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
