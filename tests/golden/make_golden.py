"""Generate the golden fixtures in this directory by running STORMM's own CPU code.

Requires the reference sources and the reference CPU build (oracle/ref/Makefile, which puts
libstormm_ref.so and stormm_ref_driver under oracle/_ref/).  Run from the repository root:

    python tests/golden/make_golden.py [--reference-root DIR]

(DIR defaults to $STORMM_REFERENCE_ROOT, else /root/reference.)

Fixtures written (numpy .npz, one per case):

* ``synthetic_<name>.npz``: synthetic molecules (the 64-atom single-point molecule and edge-case
  sizes) written as Amber prmtop/inpcrd, read back through STORMM's AtomGraph, and evaluated by
  STORMM's FP64 CPU evaluators (Potential/valence_potential.tpp, nonbonded_potential.tpp).  Each
  holds the parameters as STORMM parsed them, per-term energies and forces, GB intermediates and
  the StaticExclusionMask tables.
* ``reference_<system>_igb<k>.npz``: the reference's own test systems (Trp-cage, alanine
  dipeptide) under the settings of test/Potential/test_generalized_born.cpp:236-301, with the
  known-answer GB energies that test file asserts.
* ``synthetic_{S64,H100,O100,V100}.npz``: solvent-model variants (salt 0.15 M with dielectric
  78.5; HCT; OBC-I with dielectric 40; vacuum), run with ``--variants-only`` on its own.
* ``synthetic_N7.npz``, ``synthetic_N8.npz`` and ``reference_*_igb{7,8}.npz``
  (``--neck-only``): the neck GB models (Mongan's GBn and GBn2) on an 80-atom molecule and the
  reference systems, with the neck tables STORMM looked the pairs up in.
* ``minimize_m0.npz``: STORMM's CPU line minimizer (MolecularMechanics/minimization.tpp) on the
  64-atom molecule, energy history and final coordinates.
* ``nbwu_<case>.npz`` (``--nbwu-only``): STORMM's StaticExclusionMaskSynthesis tables and
  nonbonded work units (AtomGraphSynthesis::loadNonbondedWorkUnits) for syntheses of synthetic
  molecules; each case names its molecules by generator, seed and size, the systems per
  topology and the InitializationTask.  Small cases hold the arrays, large ones their SHA-256
  digests and sizes.
* ``charmm_ala_dipeptide.npz`` and ``charmm_dhfr.npz`` (``--charmm-only``):
  systems with CHARMM terms (one CMAP term; 2,117 Urey-Bradley terms, 418 CHARMM impropers and
  157 CMAP terms), with STORMM's energies and forces of each CHARMM term kind.
* ``restraints_r60.npz`` (``--restraints-only``): 40 constant restraints (positional, distance,
  angle and dihedral, the measured value in each region of the flat-bottom potential) on a
  60-atom molecule, STORMM's energy of each, the total and the forces.
* ``sasa_s60.npz``, ``sasa_s200.npz``, ``sasa_s33.npz`` (``--sasa-only``): STORMM's surface
  area of three synthetic molecules (272, 272 and 100 sphere points), with the points.
* ``restraint_ramps_r60.npz`` (``--ramps-only``): 24 time-dependent restraints on the same
  molecule (initial and final bounds, stiffnesses and targets, a ramp between two steps, or
  both steps equal), STORMM's energies and forces at steps before, at, within and after the
  ramps.
* ``synthetic_K64.npz`` and ``minimize_clash_k64.npz`` (``--clash-only``): a 64-atom molecule
  with close contacts (0.45 A start noise), its clash-mitigated evaluation (softened cores below
  1.5 A and below 0.9 of the pair's sigma) beside the plain one, and a minimization whose first
  25 cycles are clash-damped.
"""
from __future__ import annotations

import argparse
import os
import re
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from stormm_b200 import prmtop, synthetic  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "stormm_ref_driver")


def read_records(path):
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


def run_driver(args):
    r = subprocess.run([DRIVER] + args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver failed: {args}\n{r.stderr}")
    return r.stdout


def eval_molecule(mol, tmp, extra=()):
    top = os.path.join(tmp, mol.name + ".top")
    crd = os.path.join(tmp, mol.name + ".crd")
    out = os.path.join(tmp, mol.name + ".bin")
    prmtop.write_prmtop(mol, top)
    prmtop.write_inpcrd(mol, crd)
    run_driver(["eval", top, crd, out, "--quantize"] + list(extra))
    return read_records(out), top, crd


def gb_known_answers(ref_root):
    """Known-answer GB energies asserted by the reference's GB test (Trp-cage, DHFR, alanine
    dipeptide in that order; test/Potential/test_generalized_born.cpp:296-300)."""
    text = open(os.path.join(ref_root, "test", "Potential", "test_generalized_born.cpp")).read()
    answers = {}
    for name in ("hct", "obc", "obc2", "neck", "neck2"):
        m = re.search(r"std::vector<double> " + name + r"_gb_answer\s*=\s*\{([^}]*)\}", text)
        answers[name] = np.array([float(v) for v in m.group(1).split(",")])
    return answers


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root",
                    default=os.environ.get("STORMM_REFERENCE_ROOT", "/root/reference"))
    ap.add_argument("--variants-only", action="store_true",
                    help="write only the solvent-model variant fixtures")
    ap.add_argument("--clash-only", action="store_true",
                    help="write only the clash-damping fixtures")
    ap.add_argument("--neck-only", action="store_true",
                    help="write only the neck GB (igb 7, 8) fixtures")
    ap.add_argument("--nbwu-only", action="store_true",
                    help="write only the nonbonded work-unit fixtures")
    ap.add_argument("--charmm-only", action="store_true",
                    help="write only the CHARMM-term fixtures")
    ap.add_argument("--restraints-only", action="store_true",
                    help="write only the restraint fixture")
    ap.add_argument("--sasa-only", action="store_true",
                    help="write only the surface-area fixtures")
    ap.add_argument("--ramps-only", action="store_true",
                    help="write only the time-dependent restraint fixture")
    args = ap.parse_args()
    if not os.path.exists(DRIVER):
        raise SystemExit("build the reference driver first: make -C oracle/ref -j8")
    with tempfile.TemporaryDirectory() as tmp:
        if args.nbwu_only:
            nbwu_cases(tmp)
            return
        if args.charmm_only:
            charmm_systems(args.reference_root, tmp)
            return
        if args.ramps_only:
            ramp_case(tmp)
            return
        if args.sasa_only:
            for seed, n, npts in ((8830, 60, 272), (8840, 200, 272), (8850, 33, 100)):
                sasa_case(tmp, seed, n, npts)
            return
        if args.restraints_only:
            restraint_case(tmp)
            return
        if args.neck_only:
            for name, seed, n, igb in (("N7", 8820, 80, "7"), ("N8", 8821, 80, "8")):
                mol = synthetic.make_molecule(seed, n, noise=0.1, name=name)
                rec, _, _ = eval_molecule(mol, tmp, ["--igb", igb])
                np.savez_compressed(os.path.join(HERE, f"synthetic_{name}.npz"), **rec)
                print("wrote", name, rec["energy_terms"])
            reference_systems(args.reference_root, tmp, ((7, "neck"), (8, "neck2")))
            return
        if args.clash_only:
            mol = synthetic.make_molecule(8810, 64, noise=0.45, name="K64")
            rec, top, crd = eval_molecule(mol, tmp, ["--clash-r0", "1.5", "--clash-ratio", "0.9"])
            np.savez_compressed(os.path.join(HERE, "synthetic_K64.npz"), **rec)
            print("wrote K64", rec["energy_terms_mm"], rec["clash_energy_terms"])
            out = os.path.join(tmp, "k64_min.bin")
            run_driver(["minimize", top, crd, out, "--quantize", "--maxcyc", "60", "--ncyc", "20",
                        "--cdcyc", "25", "--clash-r0", "1.0", "--clash-ratio", "0.9"])
            mrec = read_records(out)
            np.savez_compressed(os.path.join(HERE, "minimize_clash_k64.npz"), maxcyc=60, ncyc=20,
                                cdcyc=25, clash_r0=1.0, clash_ratio=0.9, **mrec)
            print("wrote minimize_clash_k64", mrec["min_potential_history"][[0, 24, 25, -1]])
            return
        # 0. solvent-model variants of synthetic molecules: salt (Debye-Hueckel kappa) with a
        #    different dielectric, HCT, OBC-I and vacuum
        variants = (("S64", 8800, 64, ["--salt", "0.15", "--diel", "78.5"]),
                    ("H100", 8801, 100, ["--igb", "1"]),
                    ("O100", 8802, 100, ["--igb", "2", "--diel", "40"]),
                    ("V100", 8803, 100, ["--igb", "0"]))
        for name, seed, n, extra in variants:
            mol = synthetic.make_molecule(seed, n, noise=0.1, name=name)
            rec, _, _ = eval_molecule(mol, tmp, extra)
            np.savez_compressed(os.path.join(HERE, f"synthetic_{name}.npz"), **rec)
            print("wrote", name, rec["energy_terms"])
        if args.variants_only:
            return
        # 1. the single-point molecule and edge-case sizes
        mols = synthetic.workload_single()
        for n in (2, 12, 16, 17, 31, 32, 33, 48, 100, 255, 256, 257, 300):
            mols.append(synthetic.make_molecule(7700 + n, n, noise=0.1, name=f"E{n}"))
        mols.append(synthetic.make_chain(7000, 600, name="C600"))
        for mol in mols:
            rec, top, crd = eval_molecule(mol, tmp)
            np.savez_compressed(os.path.join(HERE, f"synthetic_{mol.name}.npz"), **rec)
            print("wrote", mol.name, mol.natom, rec["energy_terms"])
            if mol.name == "M0":
                out = os.path.join(tmp, "m0_min.bin")
                run_driver(["minimize", top, crd, out, "--quantize", "--maxcyc", "100",
                            "--ncyc", "50"])
                mrec = read_records(out)
                np.savez_compressed(os.path.join(HERE, "minimize_m0.npz"), maxcyc=100, ncyc=50,
                                    **mrec)
                print("wrote minimize_m0", mrec["min_potential_history"][[0, -1]])

        # 2. the reference's own GB test systems with its known answers
        reference_systems(args.reference_root, tmp, ((1, "hct"), (2, "obc"), (5, "obc2")))


def reference_systems(ref_root, tmp, models):
    """Trp-cage and alanine dipeptide under the given (igb, known-answer key) models."""
    answers = gb_known_answers(ref_root)
    tdir = os.path.join(ref_root, "test")
    systems = {"trpcage": ("trpcage.top", "trpcage.inpcrd", 1.2, 2.0, 0),
               "ala_dipeptide": ("ala_dipeptide.top", "ala_dipeptide.inpcrd", 1.2, 2.0, 2)}
    for sname, (tf, cf, scee, scnb, ans_idx) in systems.items():
        for igb, key in models:
            out = os.path.join(tmp, f"{sname}_{igb}.bin")
            run_driver(["eval", os.path.join(tdir, "Topology", tf),
                        os.path.join(tdir, "Trajectory", cf), out, "--igb", str(igb),
                        "--diel", "78.5", "--qtol", "1e-10",
                        "--qdisc", "9.31322574615478515625E-10",
                        "--scee", str(scee), "--scnb", str(scnb)])
            rec = read_records(out)
            rec["known_answer_gb"] = np.array([answers[key][ans_idx]])
            np.savez_compressed(os.path.join(HERE, f"reference_{sname}_igb{igb}.npz"), **rec)
            print("wrote", sname, igb, rec["energy_terms"][-1], answers[key][ans_idx])


def _dihedral(p0, p1, p2, p3):
    b0, b1, b2 = p1 - p0, p2 - p1, p3 - p2
    n1, n2 = np.cross(b0, b1), np.cross(b1, b2)
    return np.arctan2(np.linalg.norm(b1) * b0 @ n2, n1 @ n2)


def sasa_case(tmp, seed, n, npts):
    """STORMM's surface area (LJ-sigma radii, probe 1.4 A) of a synthetic molecule: the sphere
    points it places, the area and the energy at 0.005 kcal/mol per A^2."""
    mol = synthetic.make_molecule(seed, n, noise=0.1, name="S%d" % n)
    rec, top, crd = eval_molecule(mol, tmp)
    out = os.path.join(tmp, "sasa.bin")
    run_driver(["sasa", top, crd, str(npts), out, "--quantize"])
    rrec = read_records(out)
    rec.update({k: v for k, v in rrec.items() if k != "coords"})
    np.savez_compressed(os.path.join(HERE, "sasa_s%d.npz" % n), **rec)
    print("wrote sasa_s%d" % n, rrec["sasa_area"][0], len(rrec["sphere_points"]) // 3)


RAMP_STEPS = (0, 4, 5, 12, 17, 25, 30, 45)


def ramp_case(tmp):
    """Time-dependent restraints of every kind on the 60-atom molecule of the restraint case:
    bounds, stiffnesses and positional targets that move from initial to final values between
    two steps, plus restraints whose initial and final steps coincide (constant once engaged,
    absent before), evaluated by STORMM's CPU code at steps before, at, within and after
    every ramp."""
    mol = synthetic.make_molecule(8830, 60, noise=0.1, name="R60")
    rec, top, crd = eval_molecule(mol, tmp)
    x = rec["coords"].reshape(-1, 3)
    rng = np.random.default_rng(8831)
    rows = []
    for kind in (1, 2, 3, 4):
        for rep in range(6):
            atoms = rng.choice(mol.natom, size=4, replace=False)
            if kind == 1:
                t0 = x[atoms[0]] + rng.normal(size=3) * 1.5
                t1 = x[atoms[0]] + rng.normal(size=3) * 1.5
                value, scale = np.linalg.norm(x[atoms[0]] - t0), 1.0
            else:
                t0 = t1 = np.zeros(3)
                if kind == 2:
                    value, scale = np.linalg.norm(x[atoms[1]] - x[atoms[0]]), 1.0
                elif kind == 3:
                    ba, bc = x[atoms[0]] - x[atoms[1]], x[atoms[2]] - x[atoms[1]]
                    value = np.arccos(ba @ bc / np.linalg.norm(ba) / np.linalg.norm(bc))
                    scale = 0.5
                else:
                    value, scale = _dihedral(*x[atoms]), 0.8

            def bounds():
                off = np.sort(rng.uniform(-1.0, 1.0, size=4))
                r = [value + scale * o for o in off]
                if kind in (1, 2):
                    r = [max(v, 0.0) for v in r]
                elif kind == 3:
                    r = [min(max(v, 0.0), np.pi) for v in r]
                return r

            s0 = int(rng.choice([0, 5, 12]))
            s1 = s0 if rep == 5 else s0 + int(rng.choice([13, 18]))
            k0, k1 = rng.uniform(2.0, 30.0, size=2), rng.uniform(2.0, 30.0, size=2)
            used = list(atoms[:kind]) + [-1] * (4 - kind)
            rows.append([kind] + used + [s0, s1] + list(k0) + bounds() + list(t0) + list(k1)
                        + bounds() + list(t1))
    lst = os.path.join(tmp, "ramps.txt")
    with open(lst, "w") as f:
        for row in rows:
            f.write(" ".join(repr(float(v)) if i > 6 else str(int(v)) for i, v in enumerate(row))
                    + "\n")
    out = os.path.join(tmp, "ramps.bin")
    run_driver(["restraintramp", top, crd, lst, ",".join(map(str, RAMP_STEPS)), out,
                "--quantize"])
    rrec = read_records(out)
    rec.update({k: v for k, v in rrec.items() if k != "coords"})
    rec["restraints"] = np.array(rows, dtype=np.float64)
    rec["steps"] = np.array(RAMP_STEPS, dtype=np.int32)
    np.savez_compressed(os.path.join(HERE, "restraint_ramps_r60.npz"), **rec)
    print("wrote restraint_ramps_r60", len(rows), [float(rrec["restraint_total_%d" % s][0])
                                                   for s in RAMP_STEPS])


def restraint_case(tmp):
    """Constant restraints of every kind on a 60-atom molecule, the measured value of each
    placed in each region of the flat-bottom potential (below r1, r1-r2, r2-r3, r3-r4, above
    r4), evaluated by STORMM's CPU code."""
    mol = synthetic.make_molecule(8830, 60, noise=0.1, name="R60")
    rec, top, crd = eval_molecule(mol, tmp)
    x = rec["coords"].reshape(-1, 3)
    rng = np.random.default_rng(8830)
    # offsets of r1..r4 from the measured value that put it in region 0..4
    regions = [(0.3, 0.5, 0.7, 0.9), (-0.1, 0.2, 0.4, 0.6), (-0.3, -0.1, 0.1, 0.3),
               (-0.6, -0.4, -0.1, 0.2), (-0.9, -0.7, -0.5, -0.3)]
    rows = []
    for kind in (1, 2, 3, 4):
        for reg, off in enumerate(regions):
            for rep in range(2):
                atoms = rng.choice(mol.natom, size=4, replace=False)
                k2, k3 = rng.uniform(2.0, 30.0, size=2)
                target = np.zeros(3)
                if kind == 1:
                    target = x[atoms[0]] + rng.normal(size=3) * 1.5
                    value, scale = np.linalg.norm(x[atoms[0]] - target), 1.0
                elif kind == 2:
                    value, scale = np.linalg.norm(x[atoms[1]] - x[atoms[0]]), 1.0
                elif kind == 3:
                    ba, bc = x[atoms[0]] - x[atoms[1]], x[atoms[2]] - x[atoms[1]]
                    value = np.arccos(ba @ bc / np.linalg.norm(ba) / np.linalg.norm(bc))
                    scale = 0.5
                else:
                    value, scale = _dihedral(*x[atoms]), 0.8
                r = [value + scale * o for o in off]
                if kind in (1, 2):
                    r = [max(v, 0.0) for v in r]      # distances are not negative
                elif kind == 3:
                    r = [min(max(v, 0.0), np.pi) for v in r]
                used = list(atoms[:kind]) + [-1] * (4 - kind)
                rows.append([kind] + used + [k2, k3] + r + list(target))
    lst = os.path.join(tmp, "restraints.txt")
    with open(lst, "w") as f:
        for row in rows:
            f.write(" ".join(repr(float(v)) if i > 4 else str(int(v)) for i, v in enumerate(row))
                    + "\n")
    out = os.path.join(tmp, "restraints.bin")
    run_driver(["restraint", top, crd, lst, out, "--quantize"])
    rrec = read_records(out)
    rec.update({k: v for k, v in rrec.items() if k != "coords"})
    rec["restraints"] = np.array(rows, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "restraints_r60.npz"), **rec)
    print("wrote restraints_r60", len(rows), rrec["restraint_total"])


def charmm_systems(ref_root, tmp):
    """Systems with CHARMM terms: alanine dipeptide (one CMAP term) and dihydrofolate
    reductase (Urey-Bradley, CHARMM impropers and CMAP), OBC-II GB."""
    tdir = os.path.join(ref_root, "test")
    systems = {"ala_dipeptide": (("Topology", "ala_dipeptide.top"),
                                 ("Trajectory", "ala_dipeptide.inpcrd"),
                                 ["--scee", "1.2", "--scnb", "2.0"]),
               "dhfr": (("Topology", "dhfr_cmap.top"), ("Trajectory", "dhfr_cmap.inpcrd"), [])}
    for sname, (tf, cf, extra) in systems.items():
        out = os.path.join(tmp, f"{sname}.bin")
        run_driver(["eval", os.path.join(tdir, *tf), os.path.join(tdir, *cf), out, "--igb", "5",
                    "--diel", "78.5", "--qtol", "1e-10",
                    "--qdisc", "9.31322574615478515625E-10"] + extra)
        rec = read_records(out)
        np.savez_compressed(os.path.join(HERE, f"charmm_{sname}.npz"), **rec)
        print("wrote", sname, rec["natom"], rec["charmm_terms"], rec["charmm_terms_mm"])


# (name, [(generator, seed, natom, systems)], InitializationTask, store arrays in full)
NBWU_CASES = [
    ("mixed", [("molecule", 4101, 24, 1), ("molecule", 4102, 70, 2),
               ("molecule", 4103, 300, 3)], 3, True),
    ("edges", [("molecule", 4201, 16, 3), ("molecule", 4202, 17, 1), ("molecule", 4203, 33, 2),
               ("molecule", 4204, 64, 5), ("molecule", 4205, 250, 1)], 1, True),
    ("pair1000", [("molecule", 4301, 1000, 2)], 0, True),
    ("chains32", [("chain", 4401, 3000, 4), ("chain", 4402, 700, 3)], 5, False),
    ("chains64", [("chain", 4501, 5000, 12), ("chain", 4502, 2600, 6)], 3, False),
]


def nbwu_molecule(gen, seed, natom):
    return (synthetic.make_chain if gen == "chain" else synthetic.make_molecule)(seed, natom)


def nbwu_cases(tmp):
    import hashlib
    for name, spec, task, full in NBWU_CASES:
        lines = []
        for k, (gen, seed, natom, count) in enumerate(spec):
            top = os.path.join(tmp, f"{name}_{k}.top")
            prmtop.write_prmtop(nbwu_molecule(gen, seed, natom), top)
            lines.append(f"{top} {count}")
        lst = os.path.join(tmp, f"{name}.txt")
        with open(lst, "w") as f:
            f.write("\n".join(lines) + "\n")
        out = os.path.join(tmp, f"{name}.bin")
        run_driver(["nbwu", lst, out, "--init-task", str(task)])
        rec = read_records(out)
        keep = {"generators": np.array([s[0] for s in spec]),
                "seeds": np.array([s[1] for s in spec]), "natoms": np.array([s[2] for s in spec]),
                "counts": np.array([s[3] for s in spec]), "init_task": np.array([task]),
                "index": rec["index"]}
        for key in ("se_supertile_map_bounds", "se_supertile_map_idx", "se_tile_map_idx",
                    "se_mask_data", "nbwu_abstracts", "nbwu_insr"):
            arr = rec[key]
            if full:
                keep[key] = arr
            else:
                keep[key + "_sha256"] = np.array([hashlib.sha256(arr.tobytes()).hexdigest()])
                keep[key + "_size"] = np.array([arr.size])
        np.savez_compressed(os.path.join(HERE, f"nbwu_{name}.npz"), **keep)
        print("wrote nbwu", name, rec["nbwu_abstracts"].size // 64, "units")


if __name__ == "__main__":
    main()
