"""STORMM's valence work units (sb_valence_work_units, host only) against STORMM's own build.

The fixture (tests/golden/make_vwu_golden.py) holds, per case, the ValenceKit / ConstraintKit /
NonbondedKit arrays STORMM built from a topology and the work units buildValenceWorkUnits made
from them: Trp-cage, a DNA duplex, cAMP in water (SETTLE groups, solvent units), two drug-like
molecules, and this package's synthetic chain, molecule, two-molecule complex and a molecule
with inferred 1-4 pairs, written as prmtop files.  Every array of every unit must be equal:
import lists, manipulation masks, task counts, term lists, energy-accumulation masks and
instructions.  The atom limits STORMM's calculateValenceWorkUnitSize picks are checked the same
way."""
import os

import numpy as np
import pytest

import stormm_b200 as sb
from conftest import GOLDEN

FIXTURE = os.path.join(GOLDEN, "valence_work_units.npz")

UNIT_KEYS = {
    # fixture record: (unit key, words per item)
    "imports": ("imports", 1), "update_flags": ("update_flags", 1), "manip": ("manip", 2),
    "bond_terms": ("bond_terms", 1), "angl_terms": ("angl_terms", 1),
    "dihe_terms": ("dihe_terms", 1), "infr14_terms": ("infr14_terms", 1),
    "cbnd_terms": ("cbnd_terms", 1), "cdhe_terms": ("cdhe_terms", 2),
    "acc_bond": ("acc_bond", 1), "acc_angl": ("acc_angl", 1), "acc_dihe": ("acc_dihe", 1),
    "acc_cbnd": ("acc_cbnd", 1), "acc_cdhe": ("acc_cdhe", 1), "acc_infr14": ("acc_infr14", 1),
    "settle_insr": ("settle_insr", 2), "cgroup_insr": ("cgroup_insr", 2),
}
BOUNDS = {"imports": "imports_bounds", "update_flags": "update_flags_bounds",
          "manip": "manip_bounds", "bond_terms": "bond_terms_bounds",
          "angl_terms": "angl_terms_bounds", "dihe_terms": "dihe_terms_bounds",
          "infr14_terms": "infr14_terms_bounds", "cbnd_terms": "cbnd_terms_bounds",
          "cdhe_terms": "cdhe_terms_bounds", "acc_bond": "acc_bond_bounds",
          "acc_angl": "acc_angl_bounds", "acc_dihe": "acc_dihe_bounds",
          "acc_cbnd": "acc_cbnd_bounds", "acc_cdhe": "acc_cdhe_bounds",
          "acc_infr14": "acc_infr14_bounds", "settle_insr": "settle_insr_bounds",
          "cgroup_insr": "cgroup_insr_bounds"}
# instruction arrays without bounds records: split by the task counts
COUNTED = {"cbnd_insr": (4, 2), "angl_insr": (1, 2), "cdhe_insr": (6, 3), "infr14_insr": (8, 1)}


def _fixture():
    return dict(np.load(FIXTURE))


def _cases():
    return [str(c) for c in np.load(FIXTURE)["cases"]]


def _topology(g, case):
    r = lambda k: g[f"{case}/{k}"]
    gb = r("group_bounds")
    return {
        "natom": int(r("natom")[0]), "z_numbers": r("z_numbers"),
        "nb12_bounds": r("nb12_bounds"), "nb12_list": r("nb12x"), "solvent": r("solvent"),
        "bond_i": r("bond_i"), "bond_j": r("bond_j"), "bond_param": r("bond_param"),
        "bond_relevance": r("bond_relevance"),
        "angl_i": r("angl_i"), "angl_j": r("angl_j"), "angl_k": r("angl_k"),
        "angl_param": r("angl_param"), "angl_relevance": r("angl_relevance"),
        "dihe_i": r("dihe_i"), "dihe_j": r("dihe_j"), "dihe_k": r("dihe_k"),
        "dihe_l": r("dihe_l"), "dihe_param": r("dihe_param"), "dihe14_param": r("dihe14_param"),
        "dihe_kind": r("dihe_kind"),
        "infr14_i": r("infr14_i"), "infr14_l": r("infr14_l"), "infr14_param": r("infr14_param"),
        "settle_ox": r("settle_ox"), "settle_h1": r("settle_h1"), "settle_h2": r("settle_h2"),
        "settle_param": r("settle_param"),
        "group_bounds": gb if len(gb) > 1 else None, "group_list": r("group_list"),
        "group_param": r("group_param"), "group_param_bounds": r("group_param_bounds"),
    }


@pytest.mark.parametrize("case", _cases())
def test_units_match_stormm(case):
    g = _fixture()
    r = lambda k: g[f"{case}/{k}"]
    assert list(r("counts_ub_cimp_cmap")) == [0, 0, 0]
    units = sb.valence_work_units(_topology(g, case), int(r("atom_limit")[0]))
    assert len(units) == int(r("nunit")[0])
    tasks = r("task_counts").reshape(-1, 16)
    moved = r("moved_counts")
    offsets = {k: 0 for k in COUNTED}
    for u, unit in enumerate(units):
        np.testing.assert_array_equal(unit["task_counts"], tasks[u], err_msg=f"unit {u} tasks")
        assert unit["moved"] == moved[u]
        for rec, (key, width) in UNIT_KEYS.items():
            b = r(BOUNDS[rec])
            want = r(rec)[b[u]:b[u + 1]].astype(np.uint32 if rec != "cdhe_terms" else np.int64)
            got = np.asarray(unit[key]).reshape(-1)
            got = got.astype(np.uint32) if rec != "cdhe_terms" else got.astype(np.int64)
            np.testing.assert_array_equal(got, want, err_msg=f"{case} unit {u} {rec}")
        for rec, (task, width) in COUNTED.items():
            n = int(tasks[u][task]) * width
            want = r(rec)[offsets[rec]:offsets[rec] + n].astype(np.uint32)
            offsets[rec] += n
            np.testing.assert_array_equal(np.asarray(unit[rec]).reshape(-1), want,
                                          err_msg=f"{case} unit {u} {rec}")
    # every atom is updated by exactly one unit, and every term's energy is owned once
    nat = int(r("natom")[0])
    owners = np.zeros(nat, dtype=int)
    for unit in units:
        flags = np.unpackbits(unit["update_flags"].view(np.uint8), bitorder="little")
        owners[unit["imports"][flags[:unit["imported"]].astype(bool)]] += 1
    assert (owners == 1).all()
    for kind, n in (("bond", len(r("bond_i"))), ("angl", len(r("angl_i"))),
                    ("dihe", len(r("dihe_i"))), ("infr14", len(r("infr14_i")))):
        owned = np.zeros(n, dtype=int)
        for unit in units:
            bits = np.unpackbits(unit[f"acc_{kind}"].view(np.uint8), bitorder="little")
            terms = unit[f"{kind}_terms"]
            owned[terms[bits[:len(terms)].astype(bool)]] += 1
        assert (owned <= 1).all()


def test_unit_size_matches_stormm():
    g = _fixture()
    n = len([k for k in g if k.startswith("size_counts/")])
    for sm in (148, 132, 0):
        for k in range(n):
            lim, width = sb.valence_work_unit_size(g[f"size_counts/{k}"], sm)
            assert lim == g[f"size_sm{sm}/sizes"][k], (sm, k)
            if sm > 0:
                assert width == g[f"size_sm{sm}/widths"][k], (sm, k)


def test_bad_inputs_are_refused():
    g = _fixture()
    top = _topology(g, "trpcage_64")
    with pytest.raises(sb.StormmB200Error, match=r"\[32, 512\]"):
        sb.valence_work_units(top, 16)
    bad = dict(top)
    bad["bond_j"] = np.array(top["bond_j"]).copy()
    bad["bond_j"][3] = top["natom"]
    with pytest.raises(sb.StormmB200Error, match="outside the topology"):
        sb.valence_work_units(bad, 64)
    vs = dict(top)
    vs["z_numbers"] = np.array(top["z_numbers"]).copy()
    vs["z_numbers"][5] = 0
    with pytest.raises(sb.StormmB200Error, match="virtual sites"):
        sb.valence_work_units(vs, 64)
