// STORMM's valence work units of one topology, built on the host so a caller that keeps
// STORMM's ValenceWorkUnit tables gets them bit for bit from the same topology arrays.  The
// evaluation kernels of this library hold whole molecules per work unit and do not read these.
//
// What the reference builds (Synthesis/valence_workunit.cpp):
//   - an atom's force partners: the atom and every atom of a relevant bond or angle, of a
//     dihedral or of an inferred 1-4 pair that includes it; its movement partners: the atom and
//     every atom of a SETTLE or constraint group that includes it (findForcePartners,
//     findMovementPartners, lines 156-434);
//   - a unit grows from the first atom that no unit updates yet: a candidate atom is taken when
//     the force partners of its movement partners that the unit lacks still fit under the atom
//     limit, and the unit then updates it; the next candidates are the taken atoms' 1-2 partners
//     that no unit updates, and when none is left the unit jumps to the first atom not yet
//     updated; growth stops when no candidate of a round fits.  A topology that fits in the
//     first unit is imported whole (ValenceWorkUnit constructor, lines 863-1017);
//   - the move list is the union of the updated atoms' movement partners; the unit evaluates
//     every term that touches an atom it moves, and the first unit (in unit order) to evaluate
//     a term accumulates its energy (logActivities, lines 1963-2427);
//   - dihedrals on the same four atoms are paired into composite terms by STORMM's scan, with
//     its bounds and ownership rules reproduced as they are, and instructions are packed with
//     10-bit local atom indices and the topology's parameter indices (store*Instructions, lines
//     1149-1588).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "stormm_b200.h"
#include "synthesis.h"

struct sb_valence_units {
  struct Unit {
    int imported = 0, moved = 0, updated = 0;
    int tasks[SB_VWU_TASKS] = {};
    std::vector<int> imports, updates, moves;
    std::vector<uint32_t> manip, update_flags;
    std::vector<int> bond, angl, dihe, infr14, cbnd, cdhe;
    std::vector<uint32_t> acc_bond, acc_angl, acc_dihe, acc_cbnd, acc_cdhe, acc_infr14;
    std::vector<uint32_t> cbnd_insr, angl_insr, cdhe_insr, infr14_insr, settle_insr, cgroup_insr;
  };
  std::vector<Unit> units;
};

namespace sb {

namespace {

constexpr int kMaxVwuAtoms = 512;
constexpr int kMinVwuAtoms = kMaxVwuAtoms / 16;
enum Task { kBond = 0, kAngl, kDihe, kUbrd, kCbnd, kCimp, kCdhe, kCmap, kInfr14, kRposn, kRbond,
            kRangl, kRdihe, kVsite, kSettle, kCgroup };

int roundUp32(int x) { return ((x + 31) / 32) * 32; }

void setBit(std::vector<uint32_t> *mask, int k) { (*mask)[k >> 5] |= (1u << (k & 31)); }

bool bitSet(const uint32_t *mask, int k) { return ((mask[k >> 5] >> (k & 31)) & 1u) != 0; }

void sortUnique(std::vector<int> *v) {
  std::sort(v->begin(), v->end());
  v->erase(std::unique(v->begin(), v->end()), v->end());
}

// Items of one kind listed per atom they touch (CSR), optionally only the relevant ones
struct Touches {
  std::vector<int> bounds, items;
  void build(int natom, int nitem, std::initializer_list<const int*> atoms,
             const std::vector<char> &keep) {
    bounds.assign(natom + 1, 0);
    for (const int *col : atoms) {
      for (int t = 0; t < nitem; t++) {
        if (keep.empty() || keep[t]) bounds[col[t] + 1]++;
      }
    }
    for (int a = 0; a < natom; a++) bounds[a + 1] += bounds[a];
    items.assign(bounds[natom], 0);
    std::vector<int> fill(bounds.begin(), bounds.end() - 1);
    for (const int *col : atoms) {
      for (int t = 0; t < nitem; t++) {
        if (keep.empty() || keep[t]) items[fill[col[t]]++] = t;
      }
    }
  }
  // the items touching any atom of the list, ascending and unique
  std::vector<int> of(const std::vector<int> &atoms) const {
    std::vector<int> out;
    for (int a : atoms) out.insert(out.end(), items.begin() + bounds[a], items.begin() + bounds[a + 1]);
    sortUnique(&out);
    return out;
  }
};

class Builder {
public:
  Builder(const sb_valence_topology &t, int limit, int solvent_limit)
      : t_(t), n_(t.natom), limit_(limit), solvent_limit_(solvent_limit) {
    validate();
    std::vector<char> keep_bond(t.nbond, 1), keep_angl(t.nangl, 1);
    for (int k = 0; k < t.nbond; k++) {
      keep_bond[k] = t.bond_relevance ? bitSet(t.bond_relevance, k)
                                      : (z(t.bond_i[k]) > 0 && z(t.bond_j[k]) > 0);
    }
    for (int k = 0; k < t.nangl; k++) {
      keep_angl[k] = t.angl_relevance ? bitSet(t.angl_relevance, k)
                                      : (z(t.angl_i[k]) > 0 && z(t.angl_j[k]) > 0 &&
                                         z(t.angl_k[k]) > 0);
    }
    bonds_.build(n_, t.nbond, {t.bond_i, t.bond_j}, keep_bond);
    angls_.build(n_, t.nangl, {t.angl_i, t.angl_j, t.angl_k}, keep_angl);
    dihes_.build(n_, t.ndihe, {t.dihe_i, t.dihe_j, t.dihe_k, t.dihe_l}, {});
    infrs_.build(n_, t.ninfr14, {t.infr14_i, t.infr14_l}, {});
    setts_.build(n_, t.nsettle, {t.settle_ox, t.settle_h1, t.settle_h2}, {});
    groups_.bounds.assign(n_ + 1, 0);
    for (int g = 0; g < t.ngroup; g++) {
      for (int m = t.group_bounds[g]; m < t.group_bounds[g + 1]; m++) groups_.bounds[t.group_list[m] + 1]++;
    }
    for (int a = 0; a < n_; a++) groups_.bounds[a + 1] += groups_.bounds[a];
    groups_.items.assign(groups_.bounds[n_], 0);
    {
      std::vector<int> fill(groups_.bounds.begin(), groups_.bounds.end() - 1);
      for (int g = 0; g < t.ngroup; g++) {
        for (int m = t.group_bounds[g]; m < t.group_bounds[g + 1]; m++) {
          groups_.items[fill[t.group_list[m]]++] = g;
        }
      }
    }
    solvent_.assign(n_, 0);
    if (t.solvent != nullptr) {
      for (int a = 0; a < n_; a++) solvent_[a] = (t.solvent[a] != 0);
    }
    else {
      for (int a = 0; a < n_; a++) solvent_[a] = (t.nb12_bounds[a + 1] == t.nb12_bounds[a]);
    }
  }

  std::vector<sb_valence_units::Unit> run() {
    update_unit_.assign(n_, -1);
    stamp_.assign(n_, -1);
    first_free_ = 0;
    std::vector<sb_valence_units::Unit> units;
    while (first_free_ < n_) {
      const int lim = solvent_[first_free_] ? solvent_limit_ : limit_;
      units.emplace_back();
      grow(static_cast<int>(units.size()) - 1, lim, &units.back());
    }
    for (auto &u : units) {
      for (int a : u.updates) {
        const std::vector<int> mp = movePartners(a);
        u.moves.insert(u.moves.end(), mp.begin(), mp.end());
      }
      sortUnique(&u.moves);
      std::sort(u.imports.begin(), u.imports.end());
      std::sort(u.updates.begin(), u.updates.end());
      u.imported = static_cast<int>(u.imports.size());
      u.moved = static_cast<int>(u.moves.size());
      u.updated = static_cast<int>(u.updates.size());
      u.update_flags.assign((u.imported + 31) / 32, 0u);
      size_t p = 0;
      for (int a : u.updates) {
        while (u.imports[p] != a) p++;
        setBit(&u.update_flags, static_cast<int>(p));
      }
    }
    acc_bond_.assign(t_.nbond, -1);
    acc_angl_.assign(t_.nangl, -1);
    acc_dihe_.assign(t_.ndihe, -1);
    acc_infr_.assign(t_.ninfr14, -1);
    for (size_t k = 0; k < units.size(); k++) {
      logTerms(static_cast<int>(k), &units[k]);
    }
    return units;
  }

private:
  int z(int a) const { return t_.z_numbers ? t_.z_numbers[a] : 1; }

  void validate() const {
    const sb_valence_topology &t = t_;
    if (n_ <= 0 || t.nb12_bounds == nullptr ||
        (t.nb12_list == nullptr && t.nb12_bounds[n_] > 0)) {
      throw Error(SB_ERR_ARGUMENT, "a topology with atoms and 1-2 partner lists is required");
    }
    if (limit_ < kMinVwuAtoms || limit_ > kMaxVwuAtoms || solvent_limit_ < kMinVwuAtoms ||
        solvent_limit_ > kMaxVwuAtoms) {
      throw Error(SB_ERR_ARGUMENT, "valence work unit atom limits must lie in [32, 512]");
    }
    auto atoms = [&](int count, std::initializer_list<const int*> cols, const char *what) {
      if (count < 0) throw Error(SB_ERR_ARGUMENT, std::string("negative ") + what + " count");
      for (const int *c : cols) {
        if (count > 0 && c == nullptr) throw Error(SB_ERR_ARGUMENT, std::string(what) + " arrays missing");
        for (int k = 0; k < count; k++) {
          if (c[k] < 0 || c[k] >= n_) {
            throw Error(SB_ERR_ARGUMENT, std::string(what) + " " + std::to_string(k) +
                        " names an atom outside the topology");
          }
        }
      }
    };
    atoms(t.nbond, {t.bond_i, t.bond_j}, "bond");
    atoms(t.nangl, {t.angl_i, t.angl_j, t.angl_k}, "angle");
    atoms(t.ndihe, {t.dihe_i, t.dihe_j, t.dihe_k, t.dihe_l}, "dihedral");
    atoms(t.ninfr14, {t.infr14_i, t.infr14_l}, "inferred 1-4 pair");
    atoms(t.nsettle, {t.settle_ox, t.settle_h1, t.settle_h2}, "SETTLE group");
    auto params = [&](int count, std::initializer_list<const int*> cols, const char *what) {
      for (const int *c : cols) {
        if (count > 0 && c == nullptr) throw Error(SB_ERR_ARGUMENT, std::string(what) + " parameter indices missing");
        for (int k = 0; k < count; k++) {
          if (c[k] < 0) throw Error(SB_ERR_ARGUMENT, std::string(what) + " parameter index below zero");
        }
      }
    };
    params(t.nbond, {t.bond_param}, "bond");
    params(t.nangl, {t.angl_param}, "angle");
    params(t.ndihe, {t.dihe_param, t.dihe14_param, t.dihe_kind}, "dihedral");
    params(t.ninfr14, {t.infr14_param}, "inferred 1-4");
    params(t.nsettle, {t.settle_param}, "SETTLE");
    for (int k = 0; k < t.ndihe; k++) {
      if (t.dihe_kind[k] > 3) throw Error(SB_ERR_ARGUMENT, "dihedral kind outside 0-3");
    }
    if (t.ngroup < 0 || (t.ngroup > 0 && (t.group_bounds == nullptr || t.group_list == nullptr ||
                                         t.group_param == nullptr ||
                                         t.group_param_bounds == nullptr))) {
      throw Error(SB_ERR_ARGUMENT, "constraint group arrays missing");
    }
    for (int g = 0; g < t.ngroup; g++) {
      const int size = t.group_bounds[g + 1] - t.group_bounds[g];
      if (size < 2) throw Error(SB_ERR_ARGUMENT, "a constraint group needs two atoms or more");
      if (size - 1 >= 16) {
        throw Error(SB_ERR_ARGUMENT, "a constraint group constrains at most 15 bonds");
      }
      if (t.group_param[g] < 0) throw Error(SB_ERR_ARGUMENT, "constraint parameter index below zero");
      for (int m = t.group_bounds[g]; m < t.group_bounds[g + 1]; m++) {
        if (t.group_list[m] < 0 || t.group_list[m] >= n_) {
          throw Error(SB_ERR_ARGUMENT, "a constraint group names an atom outside the topology");
        }
      }
    }
    for (int a = 0; a < n_; a++) {
      for (int m = t.nb12_bounds[a]; m < t.nb12_bounds[a + 1]; m++) {
        if (t.nb12_list[m] < 0 || t.nb12_list[m] >= n_) {
          throw Error(SB_ERR_ARGUMENT, "a 1-2 partner outside the topology");
        }
      }
      if (z(a) == 0) {
        throw Error(SB_ERR_UNSUPPORTED, "virtual sites (atomic number 0) are not represented");
      }
    }
  }

  std::vector<int> movePartners(int a) const {
    std::vector<int> out{a};
    for (int m = setts_.bounds[a]; m < setts_.bounds[a + 1]; m++) {
      const int s = setts_.items[m];
      out.push_back(t_.settle_ox[s]);
      out.push_back(t_.settle_h1[s]);
      out.push_back(t_.settle_h2[s]);
    }
    for (int m = groups_.bounds[a]; m < groups_.bounds[a + 1]; m++) {
      const int g = groups_.items[m];
      out.insert(out.end(), t_.group_list + t_.group_bounds[g], t_.group_list + t_.group_bounds[g + 1]);
    }
    sortUnique(&out);
    return out;
  }

  void forcePartners(int a, std::vector<int> *out) const {
    out->push_back(a);
    for (int m = bonds_.bounds[a]; m < bonds_.bounds[a + 1]; m++) {
      const int k = bonds_.items[m];
      out->push_back(t_.bond_i[k]);
      out->push_back(t_.bond_j[k]);
    }
    for (int m = angls_.bounds[a]; m < angls_.bounds[a + 1]; m++) {
      const int k = angls_.items[m];
      out->push_back(t_.angl_i[k]);
      out->push_back(t_.angl_j[k]);
      out->push_back(t_.angl_k[k]);
    }
    for (int m = dihes_.bounds[a]; m < dihes_.bounds[a + 1]; m++) {
      const int k = dihes_.items[m];
      out->push_back(t_.dihe_i[k]);
      out->push_back(t_.dihe_j[k]);
      out->push_back(t_.dihe_k[k]);
      out->push_back(t_.dihe_l[k]);
    }
    for (int m = infrs_.bounds[a]; m < infrs_.bounds[a + 1]; m++) {
      const int k = infrs_.items[m];
      out->push_back(t_.infr14_i[k]);
      out->push_back(t_.infr14_l[k]);
    }
  }

  // every atom whose position the forces on a's movement partners depend on
  std::vector<int> updateDependencies(int a) const {
    std::vector<int> out;
    for (int m : movePartners(a)) forcePartners(m, &out);
    sortUnique(&out);
    return out;
  }

  void import(int u, int a, sb_valence_units::Unit *unit) {
    if (stamp_[a] == u) return;
    stamp_[a] = u;
    unit->imports.push_back(a);
  }

  void update(int u, int a, sb_valence_units::Unit *unit) {
    if (stamp_[a] != u) {
      throw Error(SB_ERR_ARGUMENT, "internal: an updated atom is not imported");
    }
    if (update_unit_[a] >= 0) return;
    update_unit_[a] = u;
    unit->updates.push_back(a);
    while (first_free_ < n_ && update_unit_[first_free_] >= 0) first_free_++;
  }

  void grow(int u, int lim, sb_valence_units::Unit *unit) {
    if (first_free_ == 0 && n_ <= lim) {
      for (int a = 0; a < n_; a++) {
        import(u, a, unit);
        update(u, a, unit);
      }
      return;
    }
    std::vector<int> cand{first_free_}, grown;
    bool full = false;
    while (!cand.empty() && !full) {
      full = true;
      grown.clear();
      for (int c : cand) {
        const std::vector<int> deps = updateDependencies(c);
        int fresh = 0;
        for (int d : deps) fresh += (stamp_[d] != u);
        if (static_cast<int>(unit->imports.size()) + fresh <= lim) {
          for (int d : deps) import(u, d, unit);
          grown.push_back(c);
          update(u, c, unit);
          full = false;
        }
      }
      cand.clear();
      for (int g : grown) {
        for (int m = t_.nb12_bounds[g]; m < t_.nb12_bounds[g + 1]; m++) {
          if (update_unit_[t_.nb12_list[m]] == -1) cand.push_back(t_.nb12_list[m]);
        }
      }
      sortUnique(&cand);
      if (cand.empty() && first_free_ < n_) cand.push_back(first_free_);
    }
  }

  static void claim(std::vector<int> *owner, int term, int u, std::vector<uint32_t> *mask, int pos) {
    if ((*owner)[term] < 0) {
      (*owner)[term] = u;
      setBit(mask, pos);
    }
  }

  // STORMM's padded length of a unit's constraint instructions: a group's bonds stay within
  // one warp-sized stretch, the stretch's rest left blank when they would cross its end
  static int paddedConstraintSlots(const std::vector<int> &group_sizes) {
    int slots = 0;
    for (int size : group_sizes) {
      const int nb = size - 1;
      if (roundUp32(slots + 1) != roundUp32(slots + nb)) slots = roundUp32(slots + 1);
      slots += nb;
    }
    return roundUp32(slots);
  }

  void logTerms(int u, sb_valence_units::Unit *unit) {
    const std::vector<int> &imp = unit->imports;
    const int base = imp.front();
    std::vector<int> local(imp.back() + 1 - base, -1);
    for (size_t i = 0; i < imp.size(); i++) local[imp[i] - base] = static_cast<int>(i);
    auto loc = [&](int a) { return static_cast<uint32_t>(local[a - base]); };
    auto words = [](size_t n) { return std::vector<uint32_t>((n + 31) / 32, 0u); };
    const sb_valence_topology &t = t_;

    unit->bond = bonds_.of(unit->moves);
    unit->acc_bond = words(unit->bond.size());
    for (size_t p = 0; p < unit->bond.size(); p++) {
      claim(&acc_bond_, unit->bond[p], u, &unit->acc_bond, static_cast<int>(p));
    }
    unit->angl = angls_.of(unit->moves);
    unit->acc_angl = words(unit->angl.size());
    for (size_t p = 0; p < unit->angl.size(); p++) {
      claim(&acc_angl_, unit->angl[p], u, &unit->acc_angl, static_cast<int>(p));
    }
    unit->dihe = dihes_.of(unit->moves);
    unit->acc_dihe = words(unit->dihe.size());
    for (size_t p = 0; p < unit->dihe.size(); p++) {
      claim(&acc_dihe_, unit->dihe[p], u, &unit->acc_dihe, static_cast<int>(p));
    }
    unit->infr14 = infrs_.of(unit->moves);
    unit->acc_infr14 = words(unit->infr14.size());
    for (size_t p = 0; p < unit->infr14.size(); p++) {
      claim(&acc_infr_, unit->infr14[p], u, &unit->acc_infr14, static_cast<int>(p));
    }
    const std::vector<int> setts = setts_.of(unit->moves);
    const std::vector<int> groups = groups_.of(unit->moves);

    // composite bonds: the bonds themselves (this path has no Urey-Bradley terms)
    unit->cbnd = unit->bond;
    unit->acc_cbnd = words(unit->cbnd.size());
    for (size_t p = 0; p < unit->cbnd.size(); p++) {
      if (acc_bond_[unit->cbnd[p]] == u) setBit(&unit->acc_cbnd, static_cast<int>(p));
    }

    // composite dihedrals: a proper dihedral is paired with a later one on the same four atoms
    // (either direction), searched between the latest first appearance and the earliest last
    // appearance of its atoms in the unit's dihedral list (that end excluded)
    const int nd = static_cast<int>(unit->dihe.size());
    std::vector<int> di(nd), dj(nd), dk(nd), dl(nd);
    std::vector<char> improper(nd), covered(nd, 0);
    std::vector<int> first_seen(imp.size(), 0), last_seen(imp.size(), 0);
    std::vector<char> seen(imp.size(), 0);
    for (int p = 0; p < nd; p++) {
      const int k = unit->dihe[p];
      di[p] = loc(t.dihe_i[k]);
      dj[p] = loc(t.dihe_j[k]);
      dk[p] = loc(t.dihe_k[k]);
      dl[p] = loc(t.dihe_l[k]);
      improper[p] = (t.dihe_kind[k] >= 2);
      for (int a : {di[p], dj[p], dk[p], dl[p]}) {
        if (seen[a]) {
          last_seen[a] = p;
        }
        else {
          first_seen[a] = p;
          seen[a] = 1;
        }
      }
    }
    std::vector<int> pos_of;     // unit dihedral position of each composite term's first member
    for (int p = 0; p < nd; p++) {
      if (t.dihe_param[unit->dihe[p]] >= 65535 || covered[p] || improper[p]) continue;
      const int lo = std::max({first_seen[di[p]], first_seen[dj[p]], first_seen[dk[p]],
                               first_seen[dl[p]], p + 1});
      const int hi = std::min({last_seen[di[p]], last_seen[dj[p]], last_seen[dk[p]],
                               last_seen[dl[p]]});
      for (int q = lo; q < hi; q++) {
        if (covered[q] || improper[q]) continue;
        const bool same = (di[q] == di[p] && dj[q] == dj[p] && dk[q] == dk[p] && dl[q] == dl[p]);
        const bool flipped = (di[q] == dl[p] && dj[q] == dk[p] && dk[q] == dj[p] && dl[q] == di[p]);
        if (same || flipped) {
          unit->cdhe.push_back(unit->dihe[p]);
          unit->cdhe.push_back(unit->dihe[q]);
          pos_of.push_back(p);
          covered[p] = covered[q] = 1;
          break;
        }
      }
    }
    for (int p = 0; p < nd; p++) {
      if (covered[p]) continue;
      unit->cdhe.push_back(unit->dihe[p]);
      unit->cdhe.push_back(-1);
      pos_of.push_back(p);
      covered[p] = 1;
    }
    const int ncdhe = static_cast<int>(pos_of.size());
    unit->acc_cdhe = words(ncdhe);
    for (int c = 0; c < ncdhe; c++) {
      // STORMM's three cases for a pair (both members owned; the lower-indexed member owned;
      // the higher-indexed one, where it tests the first member's owner again) all come down
      // to the first member's owner, as for a single dihedral
      if (acc_dihe_[unit->cdhe[2 * c]] == u) setBit(&unit->acc_cdhe, c);
    }

    // instructions, local atom indices in 10-bit fields
    for (int k : unit->cbnd) {
      unit->cbnd_insr.push_back((loc(t.bond_j[k]) << 10) | loc(t.bond_i[k]));
      unit->cbnd_insr.push_back(static_cast<uint32_t>(t.bond_param[k]));
    }
    for (int k : unit->angl) {
      unit->angl_insr.push_back((loc(t.angl_k[k]) << 20) | (loc(t.angl_j[k]) << 10) |
                                loc(t.angl_i[k]));
      unit->angl_insr.push_back(static_cast<uint32_t>(t.angl_param[k]));
    }
    for (int c = 0; c < ncdhe; c++) {
      const int p = pos_of[c];
      const int x = unit->cdhe[2 * c], y = unit->cdhe[2 * c + 1];
      uint32_t wx = (static_cast<uint32_t>(dk[p]) << 20) | (static_cast<uint32_t>(dj[p]) << 10) |
                    static_cast<uint32_t>(di[p]);
      uint32_t wy = static_cast<uint32_t>(dl[p]);
      uint32_t wz = 0u;
      if (t.dihe_kind[x] >= 2) wx |= (1u << 31);
      if (t.dihe14_param[x] >= 32) {
        throw Error(SB_ERR_UNSUPPORTED, "a dihedral's 1-4 scaling pair index exceeds 31");
      }
      wy |= static_cast<uint32_t>(t.dihe14_param[x]) << 10;
      if (y >= 0) wy |= (1u << 15);
      wy |= static_cast<uint32_t>(std::min(t.dihe_param[x], 65536)) << 16;
      if (y >= 0) {
        if (t.dihe_param[y] >= 1048576 || t.dihe14_param[y] >= 4096) {
          throw Error(SB_ERR_UNSUPPORTED, "a paired dihedral's parameter indices exceed 20 / 12 bits");
        }
        wz = static_cast<uint32_t>(t.dihe_param[y]) |
             (static_cast<uint32_t>(t.dihe14_param[y]) << 20);
      }
      unit->cdhe_insr.push_back(wx);
      unit->cdhe_insr.push_back(wy);
      unit->cdhe_insr.push_back(wz);
    }
    for (int k : unit->infr14) {
      unit->infr14_insr.push_back((loc(t.infr14_l[k]) << 10) | loc(t.infr14_i[k]) |
                                  (static_cast<uint32_t>(t.infr14_param[k]) << 20));
    }
    for (int s : setts) {
      unit->settle_insr.push_back((loc(t.settle_h2[s]) << 20) | (loc(t.settle_h1[s]) << 10) |
                                  loc(t.settle_ox[s]));
      unit->settle_insr.push_back(static_cast<uint32_t>(t.settle_param[s]));
    }
    std::vector<int> sizes;
    for (int g : groups) sizes.push_back(t.group_bounds[g + 1] - t.group_bounds[g]);
    const int slots = paddedConstraintSlots(sizes);
    unit->cgroup_insr.assign(2 * static_cast<size_t>(slots), 0u);
    int r = 0;
    for (int g : groups) {
      const int g0 = t.group_bounds[g], size = t.group_bounds[g + 1] - g0, nb = size - 1;
      const int llim = t.group_param_bounds[t.group_param[g]];
      const int stretch_end = roundUp32(r + 1);
      if (stretch_end != roundUp32(r + nb)) {
        for (; r < stretch_end; r++) {
          unit->cgroup_insr[2 * r] = static_cast<uint32_t>(r & 31) << 20;
          unit->cgroup_insr[2 * r + 1] = 0u;
        }
      }
      const uint32_t head = static_cast<uint32_t>(nb) << 28 | static_cast<uint32_t>(r & 31) << 20;
      for (int m = 1; m < size; m++, r++) {
        unit->cgroup_insr[2 * r] = head | (loc(t.group_list[g0 + m]) << 10) | loc(t.group_list[g0]);
        unit->cgroup_insr[2 * r + 1] = static_cast<uint32_t>(llim + m);
      }
    }

    int *tc = unit->tasks;
    tc[kBond] = static_cast<int>(unit->bond.size());
    tc[kAngl] = static_cast<int>(unit->angl.size());
    tc[kDihe] = nd;
    tc[kCbnd] = static_cast<int>(unit->cbnd.size());
    tc[kCdhe] = ncdhe;
    tc[kInfr14] = static_cast<int>(unit->infr14.size());
    tc[kSettle] = static_cast<int>(setts.size());
    tc[kCgroup] = slots;

    // manipulation masks: every imported atom in x, the updated ones in y, padded to 32 entries
    const int nw = (unit->imported + 31) / 32;
    unit->manip.assign(2 * static_cast<size_t>(roundUp32(nw)), 0u);
    for (int i = 0; i < unit->imported; i++) unit->manip[2 * (i >> 5)] |= (1u << (i & 31));
    for (int w = 0; w < nw; w++) unit->manip[2 * w + 1] = unit->update_flags[w];
  }

  const sb_valence_topology &t_;
  const int n_, limit_, solvent_limit_;
  Touches bonds_, angls_, dihes_, infrs_, setts_, groups_;
  std::vector<char> solvent_;
  std::vector<int> update_unit_, stamp_;
  int first_free_ = 0;
  std::vector<int> acc_bond_, acc_angl_, acc_dihe_, acc_infr_;
};

// calculateValenceWorkUnitSize for isolated systems: with SM counts, the size (32 to 512 in
// steps of 16) and kernel width of best estimated efficiency, each unit assumed to overlap its
// neighbours by 12 atoms; without, the power-of-two size of least padding
void unitSize(const int *counts, int nsys, int sm_count, int *best, int *width) {
  if (sm_count <= 0) {
    int least = 0;
    for (int vs = kMinVwuAtoms; vs <= kMaxVwuAtoms; vs *= 2) {
      const int unique = vs - 12;
      int waste = 0;
      for (int i = 0; i < nsys; i++) {
        // a system smaller than the unit sets the waste (it does not add to it)
        if (counts[i] < vs) waste = vs - counts[i];
        else waste += ((counts[i] + unique - 1) / unique) * vs - counts[i];
      }
      if (vs == kMinVwuAtoms || waste < least) {
        least = waste;
        *best = vs;
      }
    }
    return;
  }
  double total = 0.0;
  for (int i = 0; i < nsys; i++) total += counts[i];
  double best_eff = 0.0;
  const int step = kMaxVwuAtoms / 32;
  for (int vs = 2 * step; vs <= kMaxVwuAtoms; vs += step) {
    const int unique = vs - 12;
    int units = 0;
    double span = 0.0;
    for (int i = 0; i < nsys; i++) {
      if (counts[i] < vs) {
        units++;
        span += counts[i];
      }
      else {
        const int n = (counts[i] + unique - 1) / unique;
        units += n;
        span += static_cast<double>((n - 1) * vs + (counts[i] - (n - 1) * unique) + 12);
      }
    }
    const double intrinsic = total / span;
    const double mean_atoms = span / units;
    static const int kAtoms[4] = {kMaxVwuAtoms, kMaxVwuAtoms / 2, kMaxVwuAtoms / 4,
                                  kMaxVwuAtoms / 8};
    static const int kBlocksPerSm[4] = {2, 4, 8, 16};
    for (int w = 0; w < 4; w++) {
      if (vs > kAtoms[w]) continue;
      const int blocks = sm_count * kBlocksPerSm[w];
      const int rounds = (units + blocks - 1) / blocks;
      const double eff = std::sqrt(mean_atoms / kAtoms[w]) *
                         (static_cast<double>(units) / static_cast<double>(rounds * blocks)) *
                         intrinsic;
      if (eff > best_eff) {
        best_eff = eff;
        *best = vs;
        *width = w;
      }
    }
  }
}

}  // namespace

}  // namespace sb

namespace {

template <typename F> int guarded(F &&f) {
  try {
    f();
    return SB_OK;
  }
  catch (const sb::Error &e) {
    sb::setLastError(e.what());
    return e.code;
  }
  catch (const std::exception &e) {
    sb::setLastError(e.what());
    return SB_ERR_ARGUMENT;
  }
}

}  // namespace

extern "C" int sb_valence_work_units(const sb_valence_topology* top, int atom_limit,
                                     int solvent_atom_limit, sb_valence_units** out) {
  return guarded([&]() {
    if (top == nullptr || out == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "null topology or output");
    }
    *out = nullptr;
    auto set = std::make_unique<sb_valence_units>();
    set->units = sb::Builder(*top, atom_limit, solvent_atom_limit).run();
    *out = set.release();
  });
}

extern "C" int sb_valence_units_destroy(sb_valence_units* units) {
  delete units;
  return SB_OK;
}

extern "C" int sb_valence_unit_count(const sb_valence_units* units, int* count) {
  return guarded([&]() {
    if (units == nullptr || count == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null argument");
    *count = static_cast<int>(units->units.size());
  });
}

extern "C" int sb_valence_unit(const sb_valence_units* units, int unit,
                               sb_valence_unit_view* view) {
  return guarded([&]() {
    if (units == nullptr || view == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null argument");
    if (unit < 0 || unit >= static_cast<int>(units->units.size())) {
      throw sb::Error(SB_ERR_ARGUMENT, "unit index out of range");
    }
    const sb_valence_units::Unit &u = units->units[unit];
    sb_valence_unit_view v = {};
    v.imported_atoms = u.imported;
    v.moved_atoms = u.moved;
    v.updated_atoms = u.updated;
    std::copy(u.tasks, u.tasks + SB_VWU_TASKS, v.task_counts);
    v.n_manip = static_cast<int>(u.manip.size() / 2);
    v.imports = u.imports.data();
    v.manip = u.manip.data();
    v.update_flags = u.update_flags.data();
    v.bond_terms = u.bond.data();
    v.angl_terms = u.angl.data();
    v.dihe_terms = u.dihe.data();
    v.infr14_terms = u.infr14.data();
    v.cbnd_terms = u.cbnd.data();
    v.cdhe_terms = u.cdhe.data();
    v.acc_bond = u.acc_bond.data();
    v.acc_angl = u.acc_angl.data();
    v.acc_dihe = u.acc_dihe.data();
    v.acc_cbnd = u.acc_cbnd.data();
    v.acc_cdhe = u.acc_cdhe.data();
    v.acc_infr14 = u.acc_infr14.data();
    v.cbnd_insr = u.cbnd_insr.data();
    v.angl_insr = u.angl_insr.data();
    v.cdhe_insr = u.cdhe_insr.data();
    v.infr14_insr = u.infr14_insr.data();
    v.settle_insr = u.settle_insr.data();
    v.cgroup_insr = u.cgroup_insr.data();
    *view = v;
  });
}

extern "C" int sb_valence_work_unit_size(const int* atom_counts, int nsys, int sm_count,
                                         int* atom_limit, int* kernel_width) {
  return guarded([&]() {
    if (atom_counts == nullptr || nsys <= 0 || atom_limit == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "atom counts of at least one system are required");
    }
    int width = -1;
    sb::unitSize(atom_counts, nsys, sm_count, atom_limit, &width);
    if (kernel_width != nullptr && sm_count > 0) *kernel_width = width;
  });
}
