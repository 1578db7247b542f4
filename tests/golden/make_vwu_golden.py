"""Generate tests/golden/valence_work_units.npz with STORMM's own CPU build: the valence work
units buildValenceWorkUnits makes (Synthesis/valence_workunit.cpp) for topologies of STORMM's
test suite and for this package's synthetic molecules written as prmtop files, together with the
ValenceKit / ConstraintKit / NonbondedKit arrays they are built from (one synthetic molecule
lacks a quarter of its dihedrals, so STORMM infers 1-4 pairs for it); and the atom limits
calculateValenceWorkUnitSize picks for a few syntheses.

Requires the reference CPU build (oracle/ref/Makefile: oracle/_ref/stormm_ref_driver) and the
reference tree (STORMM_REFERENCE_ROOT, default /root/reference).  Run from the repository root:

    python tests/golden/make_vwu_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import DRIVER, read_records  # noqa: E402
from stormm_b200 import mmgbsa, prmtop, synthetic  # noqa: E402

REF = os.environ.get("STORMM_REFERENCE_ROOT", "/root/reference")
TOPOLOGY_DIR = os.path.join(REF, "test", "Topology")

# (case name, topology source, atom limit; 0 = STORMM's sizing for one copy on 148 SMs)
REFERENCE_CASES = [
    ("trpcage_64", "trpcage.top", 64),
    ("trpcage_auto", "trpcage.top", 0),
    ("dna_96", "dna.top", 96),
    ("camp_in_water_64", "camp_in_water.top", 64),
    ("drug_example_dry_32", "drug_example_dry.top", 32),
    ("hydrogenate_auto", "hydrogenate.top", 0),
]

SIZE_SYNTHESES = [
    [64] * 1024,
    [300] * 16,
    [2000, 3000, 4000, 5000],
    list(range(16, 257, 8)),
    [4500],
    [40] * 3 + [600],
]


def synthetic_cases():
    chain = synthetic.make_chain(synthetic._seed(6601, 0), 2000, noise=0.1, name="chain")
    mol = synthetic.make_molecule(synthetic._seed(6602, 0), 150, noise=0.1, name="mol")
    rec = synthetic.make_molecule(synthetic._seed(6603, 0), 120, noise=0.1, name="rec")
    lig = synthetic.make_molecule(synthetic._seed(6604, 0), 30, noise=0.1, name="lig")
    cpx = mmgbsa.combine(rec, lig, lig.coords + 25.0, name="cpx")
    # a quarter of the dihedrals left out: STORMM infers the 1-4 pairs they carried
    gap = synthetic.make_molecule(synthetic._seed(6605, 0), 90, noise=0.1, name="gap")
    keep = np.arange(len(gap.dihedrals)) % 4 != 0
    fields = dict(gap.__dict__)
    for k in ("dihedrals", "dihe_amp", "dihe_freq", "dihe_phase", "dihe_has14", "dihe_improper"):
        if fields.get(k) is not None:
            fields[k] = np.asarray(fields[k])[keep]
    gap = synthetic.Molecule(**fields)
    return [("chain2000_512", chain, 512), ("chain2000_128", chain, 128),
            ("mol150_auto", mol, 0), ("complex150_64", cpx, 64), ("inferred14_48", gap, 48)]


def run_case(top_path, limit):
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "vwu.bin")
        cmd = [DRIVER, "vwu", top_path, out]
        if limit > 0:
            cmd += ["--vwu-atoms", str(limit)]
        r = subprocess.run(cmd, check=True, capture_output=True, text=True)
        print(os.path.basename(top_path), r.stdout.strip())
        return read_records(out)


def main():
    arrays = {}
    names = []
    for name, top, limit in REFERENCE_CASES:
        rec = run_case(os.path.join(TOPOLOGY_DIR, top), limit)
        arrays.update({f"{name}/{k}": v for k, v in rec.items()})
        names.append(name)
    with tempfile.TemporaryDirectory() as tmp:
        for name, mol, limit in synthetic_cases():
            path = os.path.join(tmp, f"{name}.top")
            prmtop.write_prmtop(mol, path)
            rec = run_case(path, limit)
            arrays.update({f"{name}/{k}": v for k, v in rec.items()})
            names.append(name)
        lst = os.path.join(tmp, "counts.txt")
        with open(lst, "w") as f:
            f.write("\n".join(" ".join(str(c) for c in s) for s in SIZE_SYNTHESES) + "\n")
        for sm in (148, 132, 0):
            out = os.path.join(tmp, "size.bin")
            subprocess.run([DRIVER, "vwusize", lst, str(sm), out], check=True,
                           capture_output=True)
            rec = read_records(out)
            arrays[f"size_sm{sm}/sizes"] = rec["sizes"]
            arrays[f"size_sm{sm}/widths"] = rec["widths"]
    for k, s in enumerate(SIZE_SYNTHESES):
        arrays[f"size_counts/{k}"] = np.array(s, dtype=np.int32)
    arrays["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "valence_work_units.npz"), **arrays)


if __name__ == "__main__":
    main()
