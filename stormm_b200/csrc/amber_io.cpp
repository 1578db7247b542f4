// Amber topology (prmtop) and coordinate (inpcrd / ASCII restart) intake: the files STORMM's
// AtomGraph(file_name) (Topology/atomgraph.h:83,156; reader Topology/atomgraph_detailers.cpp:
// 677-1120) and PhaseSpace(file_name) read, turned into this library's sb_topology.
//
// What is read, and how it becomes an sb_topology:
//   POINTERS                       atom, type, bond / angle / dihedral counts, IFBOX
//   CHARGE                         Amber's internal units, divided by 18.2223 into electrons
//   ATOMIC_NUMBER                  optional; when absent, elements follow the nearest tabulated
//                                  mass
//   MASS, ATOM_TYPE_INDEX          Lennard-Jones type of each atom (1-based in the file)
//   NONBONDED_PARM_INDEX           type pair -> LENNARD_JONES_ACOEF / BCOEF entry, expanded into
//                                  full n_types^2 A and B tables; a negative entry is a 10-12
//                                  hydrogen-bond pair, read as zero A and B when HBOND_ACOEF /
//                                  BCOEF hold zeros there, refused otherwise
//   LENNARD_JONES_14_ACOEF / BCOEF optional (CHAMBER files), same expansion
//   BOND_*, ANGLE_*, DIHEDRAL_*    parameters by type; the *_INC_HYDROGEN and *_WITHOUT_HYDROGEN
//                                  index lists hold 3 x (atom index) and a 1-based type
//   SCEE / SCNB_SCALE_FACTOR       optional per dihedral type (1.2 / 2.0 when absent)
//   RADII, SCREEN, RADIUS_SET      intrinsic GB radii and screening factors, kept as they are
//                                  (STORMM's AtomicRadiusSet::NONE)
// A dihedral whose third atom is stored negative carries no 1-4 pair; one whose fourth atom is
// negative is improper (Amber's convention, followed by atomgraph_detailers.cpp).  1-2, 1-3 and
// 1-4 exclusions are the atoms one, two and three bonds away in the bond graph, as STORMM's
// mapExclusions (Topology/atomgraph_refinement.cpp:2735-2935) derives them; the file's
// EXCLUDED_ATOMS_LIST is not used.  A topology's unit cell (IFBOX > 0) is reported, not
// applied: this path evaluates in isolated boundary conditions.  Massless particles (virtual
// sites) are refused.  CHARMM terms (Urey-Bradley, CHARMM impropers, CMAP with its surfaces)
// are read into the topology and evaluated by the CHARMM-term kernel.
//
// sb_amber_set_implicit_solvent assigns the per-atom GB parameters the way STORMM's
// AtomGraph::setImplicitSolventModel does (Topology/atomgraph_setters.cpp:672-1060): first an
// optional radius set (Bondi, Amber6, mBondi, mBondi2, mBondi3: radii and screening factors by
// element and bonded partner; PARSE: radii), with Bondi / mBondi3 radii replacing the file's for
// the neck models when any file radius lies outside [1, 2] A; then uniform
// alpha / beta / gamma for HCT (0), OBC (0.8, 0, 2.909125) and OBC-II (1, 0.8, 4.85); for neck
// GB the uniform (1.09511284, 1.90792938, 2.50798245) with element screening factors; for neck GB
// II element alpha / beta / gamma and screening factors (parameters of Nguyen et al., J. Chem.
// Theory Comput. 9:2020, 2013, as tabulated in Constants/generalized_born.h:76-107).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "stormm_b200.h"
#include "synthesis.h"

struct sb_amber_topology {
  int natom = 0;
  int ntypes = 0;
  std::vector<double> charge, mass, lja, ljb, lja14, ljb14, pb_radii, gb_screen;
  std::vector<double> gb_alpha, gb_beta, gb_gamma;
  std::vector<int> lj_idx, z_numbers;
  std::vector<int> bond_atoms, angl_atoms, dihe_atoms, dihe_improper;
  std::vector<double> bond_keq, bond_leq, angl_keq, angl_theta0;
  std::vector<double> dihe_amp, dihe_freq, dihe_phase, dihe_scee, dihe_scnb;
  std::vector<int> excl_bounds, excl_list;
  std::vector<int> nb_bounds[3], nb_list[3];     // 1-2, 1-3, 1-4
  std::vector<std::string> atom_names, atom_types, residue_names;   // 4 characters, padded
  std::vector<int> residue_of_atom;
  std::string radius_set, title;
  int igb = -1;                                  // model applied by sb_amber_set_implicit_solvent
  int cmap_count = 0, urey_bradley_count = 0, charmm_improper_count = 0;
  // CHARMM terms, 0-based atoms, parameters expanded per term; CMAP surfaces column-major
  std::vector<int> ubrd_atoms, cimp_atoms, cmap_atoms, cmap_surface, cmap_dims;
  std::vector<double> ubrd_keq, ubrd_leq, cimp_keq, cimp_phase, cmap_values;
  int ifbox = 0;
};

namespace sb {
namespace {

constexpr double kAmberChargeScale = 18.2223;

struct Section {
  char kind = 'I';          // I, E / F (real), A (text)
  int width = 8;
  std::vector<std::string> lines;
};

std::string trimRight(const std::string &s) {
  size_t e = s.size();
  while (e > 0 && (s[e - 1] == '\r' || s[e - 1] == '\n' || s[e - 1] == ' ')) {
    e--;
  }
  return s.substr(0, e);
}

// Split a file into %FLAG sections; %COMMENT lines are skipped and %FORMAT gives the width
std::map<std::string, Section> readSections(const std::string &path) {
  std::ifstream in(path);
  if (!in) {
    throw Error(SB_ERR_ARGUMENT, "cannot open topology file " + path);
  }
  std::map<std::string, Section> out;
  std::string line;
  Section* cur = nullptr;
  bool any_flag = false;
  while (std::getline(in, line)) {
    if (line.compare(0, 5, "%FLAG") == 0) {
      std::istringstream ss(line.substr(5));
      std::string name;
      ss >> name;
      cur = &out[name];
      any_flag = true;
      continue;
    }
    if (line.compare(0, 8, "%COMMENT") == 0 || line.compare(0, 8, "%VERSION") == 0) {
      continue;
    }
    if (line.compare(0, 7, "%FORMAT") == 0) {
      if (cur == nullptr) {
        continue;
      }
      // %FORMAT(10I8), (5E16.8), (20a4), (1a80): repeat count, kind letter, field width
      size_t p = line.find('(');
      if (p == std::string::npos) {
        throw Error(SB_ERR_ARGUMENT, "malformed %FORMAT line in " + path + ": " + line);
      }
      p++;
      while (p < line.size() && std::isdigit(static_cast<unsigned char>(line[p]))) {
        p++;
      }
      if (p < line.size() && line[p] == '(') {
        p++;                                    // nested form, e.g. %FORMAT(8(F9.5))
      }
      if (p >= line.size()) {
        throw Error(SB_ERR_ARGUMENT, "malformed %FORMAT line in " + path + ": " + line);
      }
      const char k = static_cast<char>(std::toupper(static_cast<unsigned char>(line[p])));
      cur->kind = (k == 'E' || k == 'F' || k == 'D') ? 'E' : k;
      cur->width = std::atoi(line.c_str() + p + 1);
      if (cur->width <= 0) {
        throw Error(SB_ERR_ARGUMENT, "malformed %FORMAT line in " + path + ": " + line);
      }
      continue;
    }
    if (cur != nullptr) {
      cur->lines.push_back(trimRight(line));
    }
  }
  if (!any_flag) {
    throw Error(SB_ERR_ARGUMENT, path + " is not an Amber topology with %FLAG sections");
  }
  return out;
}

// Fixed-width numeric fields of a section (fields may run together, as Fortran writes them)
template <typename T> std::vector<T> numbers(const std::map<std::string, Section> &secs,
                                            const std::string &name, bool required,
                                            const std::string &path) {
  std::vector<T> out;
  auto it = secs.find(name);
  if (it == secs.end()) {
    if (required) {
      throw Error(SB_ERR_ARGUMENT, "topology " + path + " has no " + name + " section");
    }
    return out;
  }
  const Section &s = it->second;
  for (const std::string &ln : s.lines) {
    for (size_t p = 0; p < ln.size(); p += s.width) {
      std::string f = ln.substr(p, s.width);
      size_t a = f.find_first_not_of(' ');
      if (a == std::string::npos) {
        continue;
      }
      for (char &c : f) {
        if (c == 'D' || c == 'd') {
          c = 'E';
        }
      }
      char* end = nullptr;
      const double v = std::strtod(f.c_str() + a, &end);
      if (end == f.c_str() + a) {
        throw Error(SB_ERR_ARGUMENT, "unreadable field '" + f + "' in section " + name + " of " +
                    path);
      }
      out.push_back(static_cast<T>(v));
    }
  }
  return out;
}

std::string text(const std::map<std::string, Section> &secs, const std::string &name) {
  auto it = secs.find(name);
  if (it == secs.end()) {
    return std::string();
  }
  std::string out;
  for (const std::string &ln : it->second.lines) {
    out += ln;
  }
  size_t a = out.find_first_not_of(' ');
  return (a == std::string::npos) ? std::string() : trimRight(out.substr(a));
}

// Fixed-width text fields (atom names, types, residue labels), padded to the field width
std::vector<std::string> words(const std::map<std::string, Section> &secs,
                               const std::string &name) {
  std::vector<std::string> out;
  auto it = secs.find(name);
  if (it == secs.end()) {
    return out;
  }
  const int w = it->second.width;
  for (std::string ln : it->second.lines) {
    if (ln.empty()) {
      continue;
    }
    ln.resize(((ln.size() + w - 1) / w) * w, ' ');
    for (size_t p = 0; p < ln.size(); p += w) {
      out.push_back(ln.substr(p, w));
    }
  }
  return out;
}

void needCount(size_t have, size_t want, const std::string &what, const std::string &path) {
  if (have < want) {
    throw Error(SB_ERR_ARGUMENT, "topology " + path + ": section " + what + " holds " +
                std::to_string(have) + " values, " + std::to_string(want) + " expected");
  }
}

// Element of a mass when ATOMIC_NUMBER is absent: the nearest of a few common elements
int elementOfMass(double m) {
  static const double masses[] = {1.008, 4.003, 6.94, 12.011, 14.007, 15.999, 18.998, 22.990,
                                  24.305, 30.974, 32.06, 35.45, 39.098, 40.078, 55.845, 65.38,
                                  79.904, 126.904};
  static const int znum[] = {1, 2, 3, 6, 7, 8, 9, 11, 12, 15, 16, 17, 19, 20, 26, 30, 35, 53};
  int best = 0;
  for (int k = 1; k < static_cast<int>(sizeof(znum) / sizeof(int)); k++) {
    if (std::fabs(m - masses[k]) < std::fabs(m - masses[best])) {
      best = k;
    }
  }
  return (m > 0.5) ? znum[best] : 0;
}

// Atoms one, two and three bonds away from each atom (excluding atoms already nearer)
void bondGraphExclusions(sb_amber_topology* t) {
  const int n = t->natom;
  std::vector<std::vector<int>> adj(n);
  const int nb = static_cast<int>(t->bond_atoms.size() / 2);
  for (int b = 0; b < nb; b++) {
    const int i = t->bond_atoms[2 * b], j = t->bond_atoms[2 * b + 1];
    if (i == j) {
      continue;
    }
    adj[i].push_back(j);
    adj[j].push_back(i);
  }
  std::vector<int> dist(n, -1);
  std::vector<int> touched;
  std::vector<std::vector<int>> lists[3];
  for (int lv = 0; lv < 3; lv++) {
    lists[lv].assign(n, std::vector<int>());
  }
  for (int a = 0; a < n; a++) {
    dist[a] = 0;
    touched.assign(1, a);
    std::vector<int> frontier(1, a);
    for (int lv = 1; lv <= 3; lv++) {
      std::vector<int> next;
      for (int u : frontier) {
        for (int v : adj[u]) {
          if (dist[v] < 0) {
            dist[v] = lv;
            touched.push_back(v);
            next.push_back(v);
            lists[lv - 1][a].push_back(v);
          }
        }
      }
      frontier.swap(next);
    }
    for (int v : touched) {
      dist[v] = -1;
    }
  }
  t->excl_bounds.assign(n + 1, 0);
  t->excl_list.clear();
  for (int lv = 0; lv < 3; lv++) {
    t->nb_bounds[lv].assign(n + 1, 0);
    t->nb_list[lv].clear();
  }
  for (int a = 0; a < n; a++) {
    std::vector<int> all;
    for (int lv = 0; lv < 3; lv++) {
      std::vector<int> &l = lists[lv][a];
      std::sort(l.begin(), l.end());
      t->nb_list[lv].insert(t->nb_list[lv].end(), l.begin(), l.end());
      t->nb_bounds[lv][a + 1] = static_cast<int>(t->nb_list[lv].size());
      all.insert(all.end(), l.begin(), l.end());
    }
    std::sort(all.begin(), all.end());
    t->excl_list.insert(t->excl_list.end(), all.begin(), all.end());
    t->excl_bounds[a + 1] = static_cast<int>(t->excl_list.size());
  }
}

void expandLennardJones(const std::vector<int> &parm_index, const std::vector<double> &acoef,
                        const std::vector<double> &bcoef, const std::vector<double> &hb_a,
                        const std::vector<double> &hb_b, int ntypes, std::vector<double>* lja,
                        std::vector<double>* ljb, const std::string &what,
                        const std::string &path) {
  lja->assign(static_cast<size_t>(ntypes) * ntypes, 0.0);
  ljb->assign(static_cast<size_t>(ntypes) * ntypes, 0.0);
  for (int i = 0; i < ntypes; i++) {
    for (int j = 0; j < ntypes; j++) {
      const int ico = parm_index[static_cast<size_t>(ntypes) * i + j];
      if (ico > 0) {
        if (ico > static_cast<int>(acoef.size()) || ico > static_cast<int>(bcoef.size())) {
          throw Error(SB_ERR_ARGUMENT, "topology " + path + ": " + what +
                      " index past the end of its coefficient tables");
        }
        (*lja)[static_cast<size_t>(ntypes) * i + j] = acoef[ico - 1];
        (*ljb)[static_cast<size_t>(ntypes) * i + j] = bcoef[ico - 1];
      }
      else if (ico < 0) {
        const int h = -ico - 1;
        const bool zero = (h >= static_cast<int>(hb_a.size()) || hb_a[h] == 0.0) &&
                          (h >= static_cast<int>(hb_b.size()) || hb_b[h] == 0.0);
        if (!zero) {
          throw Error(SB_ERR_UNSUPPORTED, "topology " + path + " uses 10-12 hydrogen-bond "
                      "terms, which this library does not evaluate");
        }
      }
    }
  }
}

sb_amber_topology* readTopology(const std::string &path) {
  const std::map<std::string, Section> secs = readSections(path);
  const std::vector<int> ptr = numbers<int>(secs, "POINTERS", true, path);
  needCount(ptr.size(), 20, "POINTERS", path);
  auto t = new sb_amber_topology();
  try {
    const int n = ptr[0];
    const int ntypes = ptr[1];
    const int nbonh = ptr[2], mbona = ptr[3], ntheth = ptr[4], mtheta = ptr[5];
    const int nphih = ptr[6], mphia = ptr[7];
    const int nptra = ptr[17];
    if (n <= 0 || ntypes <= 0) {
      throw Error(SB_ERR_ARGUMENT, "topology " + path + " declares no atoms or no atom types");
    }
    // a unit cell (IFBOX > 0) is recorded, not applied: this path evaluates every system in
    // isolated boundary conditions, as STORMM's GB evaluation of such a topology does
    t->ifbox = (ptr.size() > 27) ? ptr[27] : 0;
    t->natom = n;
    t->ntypes = ntypes;
    t->title = text(secs, "TITLE");
    t->radius_set = text(secs, "RADIUS_SET");

    std::vector<double> q = numbers<double>(secs, "CHARGE", true, path);
    needCount(q.size(), n, "CHARGE", path);
    t->charge.resize(n);
    for (int i = 0; i < n; i++) {
      t->charge[i] = q[i] / kAmberChargeScale;
    }
    t->mass = numbers<double>(secs, "MASS", true, path);
    needCount(t->mass.size(), n, "MASS", path);
    t->mass.resize(n);
    for (int i = 0; i < n; i++) {
      if (!(t->mass[i] > 1.0e-6)) {
        throw Error(SB_ERR_UNSUPPORTED, "topology " + path + " holds massless particles "
                    "(virtual sites), which this path does not evaluate");
      }
    }
    t->z_numbers = numbers<int>(secs, "ATOMIC_NUMBER", false, path);
    if (t->z_numbers.empty()) {
      t->z_numbers.resize(n);
      for (int i = 0; i < n; i++) {
        t->z_numbers[i] = elementOfMass(t->mass[i]);
      }
    }
    needCount(t->z_numbers.size(), n, "ATOMIC_NUMBER", path);
    t->z_numbers.resize(n);

    t->lj_idx = numbers<int>(secs, "ATOM_TYPE_INDEX", true, path);
    needCount(t->lj_idx.size(), n, "ATOM_TYPE_INDEX", path);
    t->lj_idx.resize(n);
    for (int i = 0; i < n; i++) {
      t->lj_idx[i] -= 1;
      if (t->lj_idx[i] < 0 || t->lj_idx[i] >= ntypes) {
        throw Error(SB_ERR_ARGUMENT, "topology " + path + ": atom type index out of range");
      }
    }
    const std::vector<int> parm = numbers<int>(secs, "NONBONDED_PARM_INDEX", true, path);
    needCount(parm.size(), static_cast<size_t>(ntypes) * ntypes, "NONBONDED_PARM_INDEX", path);
    const std::vector<double> hb_a = numbers<double>(secs, "HBOND_ACOEF", false, path);
    const std::vector<double> hb_b = numbers<double>(secs, "HBOND_BCOEF", false, path);
    expandLennardJones(parm, numbers<double>(secs, "LENNARD_JONES_ACOEF", true, path),
                       numbers<double>(secs, "LENNARD_JONES_BCOEF", true, path), hb_a, hb_b,
                       ntypes, &t->lja, &t->ljb, "LENNARD_JONES", path);
    if (secs.count("LENNARD_JONES_14_ACOEF") != 0) {
      expandLennardJones(parm, numbers<double>(secs, "LENNARD_JONES_14_ACOEF", true, path),
                         numbers<double>(secs, "LENNARD_JONES_14_BCOEF", true, path), hb_a, hb_b,
                         ntypes, &t->lja14, &t->ljb14, "LENNARD_JONES_14", path);
    }

    // Names, types and residues: only the radius sets look at them
    t->atom_names = words(secs, "ATOM_NAME");
    t->atom_types = words(secs, "AMBER_ATOM_TYPE");
    t->atom_names.resize(n, std::string(4, ' '));
    t->atom_types.resize(n, std::string(4, ' '));
    const std::vector<std::string> labels = words(secs, "RESIDUE_LABEL");
    const std::vector<int> rptr = numbers<int>(secs, "RESIDUE_POINTER", false, path);
    t->residue_of_atom.assign(n, 0);
    for (size_t r = 0; r < rptr.size(); r++) {
      const int first = rptr[r] - 1;
      const int last = (r + 1 < rptr.size()) ? rptr[r + 1] - 1 : n;
      for (int a = std::max(first, 0); a < std::min(last, n); a++) {
        t->residue_of_atom[a] = static_cast<int>(r);
      }
    }
    t->residue_names = labels;
    if (t->residue_names.empty()) {
      t->residue_names.assign(1, std::string(4, ' '));
    }
    for (int a = 0; a < n; a++) {
      if (t->residue_of_atom[a] >= static_cast<int>(t->residue_names.size())) {
        t->residue_of_atom[a] = 0;
      }
    }

    // Bonds
    const std::vector<double> bk = numbers<double>(secs, "BOND_FORCE_CONSTANT", true, path);
    const std::vector<double> br = numbers<double>(secs, "BOND_EQUIL_VALUE", true, path);
    for (const char* name : {"BONDS_INC_HYDROGEN", "BONDS_WITHOUT_HYDROGEN"}) {
      const std::vector<int> v = numbers<int>(secs, name, true, path);
      needCount(v.size(), 3 * static_cast<size_t>(name[6] == 'I' ? nbonh : mbona), name, path);
      const int cnt = (name[6] == 'I') ? nbonh : mbona;
      for (int b = 0; b < cnt; b++) {
        const int i = std::abs(v[3 * b]) / 3, j = std::abs(v[3 * b + 1]) / 3;
        const int ty = v[3 * b + 2] - 1;
        if (i >= n || j >= n || ty < 0 || ty >= static_cast<int>(std::min(bk.size(), br.size()))) {
          throw Error(SB_ERR_ARGUMENT, "topology " + path + ": bond index out of range");
        }
        t->bond_atoms.push_back(i);
        t->bond_atoms.push_back(j);
        t->bond_keq.push_back(bk[ty]);
        t->bond_leq.push_back(br[ty]);
      }
    }

    // Angles
    const std::vector<double> ak = numbers<double>(secs, "ANGLE_FORCE_CONSTANT", true, path);
    const std::vector<double> at = numbers<double>(secs, "ANGLE_EQUIL_VALUE", true, path);
    for (const char* name : {"ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN"}) {
      const bool inc = (name[7] == 'I');
      const int cnt = inc ? ntheth : mtheta;
      const std::vector<int> v = numbers<int>(secs, name, true, path);
      needCount(v.size(), 4 * static_cast<size_t>(cnt), name, path);
      for (int a = 0; a < cnt; a++) {
        const int i = std::abs(v[4 * a]) / 3, j = std::abs(v[4 * a + 1]) / 3;
        const int k = std::abs(v[4 * a + 2]) / 3, ty = v[4 * a + 3] - 1;
        if (i >= n || j >= n || k >= n || ty < 0 ||
            ty >= static_cast<int>(std::min(ak.size(), at.size()))) {
          throw Error(SB_ERR_ARGUMENT, "topology " + path + ": angle index out of range");
        }
        t->angl_atoms.insert(t->angl_atoms.end(), {i, j, k});
        t->angl_keq.push_back(ak[ty]);
        t->angl_theta0.push_back(at[ty]);
      }
    }

    // Dihedrals
    const std::vector<double> dk = numbers<double>(secs, "DIHEDRAL_FORCE_CONSTANT", true, path);
    const std::vector<double> dn = numbers<double>(secs, "DIHEDRAL_PERIODICITY", true, path);
    const std::vector<double> dp = numbers<double>(secs, "DIHEDRAL_PHASE", true, path);
    std::vector<double> scee = numbers<double>(secs, "SCEE_SCALE_FACTOR", false, path);
    std::vector<double> scnb = numbers<double>(secs, "SCNB_SCALE_FACTOR", false, path);
    const size_t ndty = std::min(dk.size(), std::min(dn.size(), dp.size()));
    if (ndty < static_cast<size_t>(nptra)) {
      throw Error(SB_ERR_ARGUMENT, "topology " + path + ": dihedral parameter tables are short");
    }
    if (scee.size() < ndty) {
      scee.resize(ndty, 1.2);
    }
    if (scnb.size() < ndty) {
      scnb.resize(ndty, 2.0);
    }
    for (const char* name : {"DIHEDRALS_INC_HYDROGEN", "DIHEDRALS_WITHOUT_HYDROGEN"}) {
      const bool inc = (name[10] == 'I');
      const int cnt = inc ? nphih : mphia;
      const std::vector<int> v = numbers<int>(secs, name, true, path);
      needCount(v.size(), 5 * static_cast<size_t>(cnt), name, path);
      for (int d = 0; d < cnt; d++) {
        const int* e = &v[5 * d];
        const int i = std::abs(e[0]) / 3, j = std::abs(e[1]) / 3;
        const int k = std::abs(e[2]) / 3, l = std::abs(e[3]) / 3, ty = e[4] - 1;
        if (i >= n || j >= n || k >= n || l >= n || ty < 0 || ty >= static_cast<int>(ndty)) {
          throw Error(SB_ERR_ARGUMENT, "topology " + path + ": dihedral index out of range");
        }
        const bool has14 = (e[2] >= 0);
        t->dihe_atoms.insert(t->dihe_atoms.end(), {i, j, k, l});
        t->dihe_amp.push_back(dk[ty]);
        t->dihe_freq.push_back(dn[ty]);
        t->dihe_phase.push_back(dp[ty]);
        t->dihe_scee.push_back(has14 ? scee[ty] : 0.0);
        t->dihe_scnb.push_back(has14 ? scnb[ty] : 0.0);
        t->dihe_improper.push_back(e[3] < 0 ? 1 : 0);
      }
    }

    // Implicit solvent parameters as the file holds them
    t->pb_radii = numbers<double>(secs, "RADII", false, path);
    t->gb_screen = numbers<double>(secs, "SCREEN", false, path);
    t->pb_radii.resize(n, 0.0);
    t->gb_screen.resize(n, 0.0);

    // CHARMM terms (Topology/atomgraph_detailers.cpp:897-990, 1196-1240): 1-based atoms, each
    // term's last entry its 1-based parameter set; CMAP surfaces are stored phi-major and kept
    // here column-major (phi index fastest), as the evaluation indexes them
    auto atom0 = [&](int v) {
      if (v < 1 || v > n) throw Error(SB_ERR_ARGUMENT, path + ": CHARMM term atom out of range");
      return v - 1;
    };
    const std::vector<int> ub = numbers<int>(secs, "CHARMM_UREY_BRADLEY_COUNT", false, path);
    t->urey_bradley_count = ub.empty() ? 0 : ub[0];
    if (t->urey_bradley_count > 0) {
      const std::vector<int> a = numbers<int>(secs, "CHARMM_UREY_BRADLEY", true, path);
      const std::vector<double> k = numbers<double>(secs, "CHARMM_UREY_BRADLEY_FORCE_CONSTANT",
                                                    true, path);
      const std::vector<double> r = numbers<double>(secs, "CHARMM_UREY_BRADLEY_EQUIL_VALUE",
                                                    true, path);
      if (a.size() < 3 * static_cast<size_t>(t->urey_bradley_count)) {
        throw Error(SB_ERR_ARGUMENT, path + ": short CHARMM_UREY_BRADLEY section");
      }
      for (int q = 0; q < t->urey_bradley_count; q++) {
        const int p = a[3 * q + 2] - 1;
        if (p < 0 || p >= static_cast<int>(std::min(k.size(), r.size()))) {
          throw Error(SB_ERR_ARGUMENT, path + ": Urey-Bradley parameter index out of range");
        }
        t->ubrd_atoms.push_back(atom0(a[3 * q]));
        t->ubrd_atoms.push_back(atom0(a[3 * q + 1]));
        t->ubrd_keq.push_back(k[p]);
        t->ubrd_leq.push_back(r[p]);
      }
    }
    const std::vector<int> ci = numbers<int>(secs, "CHARMM_NUM_IMPROPERS", false, path);
    t->charmm_improper_count = ci.empty() ? 0 : ci[0];
    if (t->charmm_improper_count > 0) {
      const std::vector<int> a = numbers<int>(secs, "CHARMM_IMPROPERS", true, path);
      const std::vector<double> k = numbers<double>(secs, "CHARMM_IMPROPER_FORCE_CONSTANT", true,
                                                    path);
      const std::vector<double> ph = numbers<double>(secs, "CHARMM_IMPROPER_PHASE", true, path);
      if (a.size() < 5 * static_cast<size_t>(t->charmm_improper_count)) {
        throw Error(SB_ERR_ARGUMENT, path + ": short CHARMM_IMPROPERS section");
      }
      for (int q = 0; q < t->charmm_improper_count; q++) {
        const int p = a[5 * q + 4] - 1;
        if (p < 0 || p >= static_cast<int>(std::min(k.size(), ph.size()))) {
          throw Error(SB_ERR_ARGUMENT, path + ": CHARMM improper parameter index out of range");
        }
        for (int m = 0; m < 4; m++) t->cimp_atoms.push_back(atom0(a[5 * q + m]));
        t->cimp_keq.push_back(k[p]);
        t->cimp_phase.push_back(ph[p]);
      }
    }
    for (const std::string prefix : {"CHARMM_CMAP_", "CMAP_"}) {
      const std::vector<int> cm = numbers<int>(secs, prefix + "COUNT", false, path);
      if (cm.empty()) continue;
      t->cmap_count = cm[0];
      const int nsurf = (cm.size() > 1) ? cm[1] : 0;
      if (t->cmap_count <= 0) break;
      t->cmap_dims = numbers<int>(secs, prefix + "RESOLUTION", true, path);
      if (nsurf <= 0 || static_cast<int>(t->cmap_dims.size()) < nsurf) {
        throw Error(SB_ERR_ARGUMENT, path + ": CMAP surfaces without resolutions");
      }
      t->cmap_dims.resize(nsurf);
      for (int sfc = 0; sfc < nsurf; sfc++) {
        const int dim = t->cmap_dims[sfc];
        const std::string flag = prefix + "PARAMETER_" + (sfc + 1 < 10 ? "0" : "") +
                                 std::to_string(sfc + 1);
        const std::vector<double> grid = numbers<double>(secs, flag, true, path);
        if (dim < 1 || grid.size() < static_cast<size_t>(dim) * dim) {
          throw Error(SB_ERR_ARGUMENT, path + ": short " + flag + " section");
        }
        for (int k = 0; k < dim; k++) {
          for (int j = 0; j < dim; j++) {
            t->cmap_values.push_back(grid[static_cast<size_t>(j) * dim + k]);
          }
        }
      }
      const std::vector<int> a = numbers<int>(secs, prefix + "INDEX", true, path);
      if (a.size() < 6 * static_cast<size_t>(t->cmap_count)) {
        throw Error(SB_ERR_ARGUMENT, path + ": short " + prefix + "INDEX section");
      }
      for (int q = 0; q < t->cmap_count; q++) {
        for (int m = 0; m < 5; m++) t->cmap_atoms.push_back(atom0(a[6 * q + m]));
        const int sfc = a[6 * q + 5] - 1;
        if (sfc < 0 || sfc >= nsurf) {
          throw Error(SB_ERR_ARGUMENT, path + ": CMAP surface index out of range");
        }
        t->cmap_surface.push_back(sfc);
      }
      break;
    }

    bondGraphExclusions(t);
    return t;
  }
  catch (...) {
    delete t;
    throw;
  }
}

// Intrinsic radii and screening factors of a radius set, by element with the bonded-partner,
// united-atom and residue rules of Amber's radius sets as STORMM's
// AtomGraph::setImplicitSolventModel applies them (Topology/atomgraph_setters.cpp:743-958)
void applyRadiusSet(sb_amber_topology* t, int set) {
  const int n = t->natom;
  const std::vector<int> &z = t->z_numbers;
  const std::vector<int> &b12 = t->nb_bounds[0], &x12 = t->nb_list[0];
  const std::vector<int> &b13 = t->nb_bounds[1], &x13 = t->nb_list[1];
  const bool bondi_family = (set == SB_RADII_BONDI || set == SB_RADII_AMBER6 ||
                             set == SB_RADII_MBONDI || set == SB_RADII_MBONDI2 ||
                             set == SB_RADII_MBONDI3);
  for (int i = 0; i < n; i++) {
    double rad = t->pb_radii[i];
    const std::string &res = t->residue_names[t->residue_of_atom[i]];
    const std::string &name = t->atom_names[i];
    if (bondi_family) {
      switch (z[i]) {
      case 1:
        rad = 1.2;
        if (b12[i + 1] > b12[i]) {
          const int partner = x12[b12[i]];
          if (set == SB_RADII_AMBER6 || set == SB_RADII_MBONDI) {
            switch (z[partner]) {
            case 1:
              if ((t->atom_types[partner][0] == 'H' || t->atom_types[partner][0] == 'h') &&
                  (t->atom_types[partner][1] == 'W' || t->atom_types[partner][1] == 'w')) {
                rad = 0.8;
              }
              break;
            case 6:
              rad = 1.3;
              break;
            case 7:
              if (set == SB_RADII_MBONDI) {
                rad = 1.3;
              }
              break;
            case 8:
            case 16:
              rad = 0.8;
              break;
            default:
              break;
            }
          }
          else if ((set == SB_RADII_MBONDI2 || set == SB_RADII_MBONDI3) && z[partner] == 7) {
            rad = 1.3;
            if (set == SB_RADII_MBONDI3 && t->residue_names[t->residue_of_atom[partner]] ==
                "ARG " && name[0] == 'H' && (name[1] == 'H' || name[1] == 'E')) {
              rad = 1.17;
            }
          }
        }
        break;
      case 6: {
        // united-atom carbons (types C1 / C2 / C3 carrying the mass of their hydrogens), with
        // repartitioned hydrogen mass returned to the carbon first
        double m = t->mass[i];
        for (int k = b12[i]; k < b12[i + 1]; k++) {
          if (z[x12[k]] == 1 && t->mass[x12[k]] > 1.008) {
            m += t->mass[x12[k]] - 1.008;
          }
        }
        const std::string &ty = t->atom_types[i];
        const bool united = (ty[0] == 'C' && ((ty[1] == '1' && m > 13.018) ||
                                              (ty[1] == '2' && m > 14.026) ||
                                              (ty[1] == '3' && m > 15.034)));
        rad = united ? 2.2 : 1.7;
        break;
      }
      case 7:
        rad = 1.55;
        break;
      case 8:
        rad = 1.5;
        if (set == SB_RADII_MBONDI3) {
          if (((res == "ASP " || res == "AS4 ") && (name == "OD1 " || name == "OD2 ")) ||
              ((res == "GLU " || res == "GL4 ") && (name == "OE1 " || name == "OE2 ")) ||
              name == "OXT ") {
            rad = 1.4;
          }
          if (b12[i + 1] - b12[i] == 1 && z[x12[b12[i]]] == 6) {
            for (int k = b13[i]; k < b13[i + 1]; k++) {
              if (z[x13[k]] == 8) {
                rad = 1.4;
              }
            }
          }
        }
        break;
      case 9: rad = 1.5; break;
      case 14: rad = 2.1; break;
      case 15: rad = 1.85; break;
      case 16: rad = 1.8; break;
      case 17: rad = 1.7; break;
      default: rad = 1.5; break;
      }
      double screen = 0.8;
      switch (z[i]) {
      case 1: screen = 0.85; break;
      case 6: screen = 0.72; break;
      case 7: screen = 0.79; break;
      case 8: screen = 0.85; break;
      case 9: screen = 0.88; break;
      case 15: screen = 0.86; break;
      case 16: screen = 0.96; break;
      default: break;
      }
      t->gb_screen[i] = screen;
    }
    else if (set == SB_RADII_PARSE) {
      switch (z[i]) {
      case 1: rad = 1.0; break;
      case 6: rad = 1.7; break;
      case 7: rad = 1.5; break;
      case 8: rad = 1.4; break;
      case 16: rad = 1.85; break;
      default: rad = 1.5; break;
      }
    }
    t->pb_radii[i] = rad;
  }
}

void setImplicitSolvent(sb_amber_topology* t, int igb, int radius_set) {
  const int n = t->natom;
  if (igb != SB_GB_NONE && igb != SB_GB_HCT && igb != SB_GB_OBC && igb != SB_GB_OBC2 &&
      igb != SB_GB_NECK && igb != SB_GB_NECK2) {
    throw Error(SB_ERR_ARGUMENT, "unknown GB model " + std::to_string(igb));
  }
  if (radius_set < SB_RADII_NONE || radius_set > SB_RADII_PARSE) {
    throw Error(SB_ERR_ARGUMENT, "unknown radius set " + std::to_string(radius_set));
  }
  // The neck models need every radius in [1, 2] A: otherwise Bondi radii (neck GB) or mBondi3
  // radii (neck GB II) replace the file's, as in STORMM
  if ((igb == SB_GB_NECK && radius_set != SB_RADII_BONDI) ||
      (igb == SB_GB_NECK2 && radius_set != SB_RADII_MBONDI3)) {
    bool bad = false;
    for (int i = 0; i < n; i++) {
      bad = bad || t->pb_radii[i] < 1.0 || t->pb_radii[i] > 2.0;
    }
    if (bad) {
      radius_set = (igb == SB_GB_NECK) ? SB_RADII_BONDI : SB_RADII_MBONDI3;
    }
  }
  if (igb != SB_GB_NONE) {
    applyRadiusSet(t, radius_set);
  }
  t->gb_alpha.assign(n, 0.0);
  t->gb_beta.assign(n, 0.0);
  t->gb_gamma.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    const int z = t->z_numbers[i];
    double a = 0.0, b = 0.0, g = 0.0;
    switch (igb) {
    case SB_GB_OBC:
      a = 0.8; b = 0.0; g = 2.909125;
      break;
    case SB_GB_OBC2:
      a = 1.0; b = 0.8; g = 4.85;
      break;
    case SB_GB_NECK:
      a = 1.09511284; b = 1.90792938; g = 2.50798245;
      switch (z) {
      case 1: t->gb_screen[i] = 1.09085413633; break;
      case 6: t->gb_screen[i] = 0.484353823306; break;
      case 7: t->gb_screen[i] = 0.700147318409; break;
      case 8: t->gb_screen[i] = 1.06557401132; break;
      case 16: t->gb_screen[i] = 0.602256336067; break;
      default: t->gb_screen[i] = 0.5; break;
      }
      break;
    case SB_GB_NECK2:
      switch (z) {
      case 1: a = 0.788440; b = 0.798699; g = 0.437334; t->gb_screen[i] = 1.425952; break;
      case 6: a = 0.733756; b = 0.506378; g = 0.205844; t->gb_screen[i] = 1.058554; break;
      case 7: a = 0.503364; b = 0.316828; g = 0.192915; t->gb_screen[i] = 0.733599; break;
      case 8: a = 0.867814; b = 0.876635; g = 0.387882; t->gb_screen[i] = 1.061039; break;
      case 15: a = 1.0; b = 0.8; g = 4.85; t->gb_screen[i] = 0.5; break;
      case 16: a = 0.867814; b = 0.876635; g = 0.387882; t->gb_screen[i] = -0.703469; break;
      default: a = 1.0; b = 0.8; g = 4.85; t->gb_screen[i] = 0.5; break;
      }
      break;
    default:
      break;
    }
    t->gb_alpha[i] = a;
    t->gb_beta[i] = b;
    t->gb_gamma[i] = g;
  }
  t->igb = igb;
}

void fillView(const sb_amber_topology* t, sb_amber_view* v) {
  sb_topology &s = v->topology;
  s = sb_topology();
  s.natom = t->natom;
  s.charge = t->charge.data();
  s.lj_idx = t->lj_idx.data();
  s.n_lj_types = t->ntypes;
  s.lja = t->lja.data();
  s.ljb = t->ljb.data();
  s.lja14 = t->lja14.empty() ? nullptr : t->lja14.data();
  s.ljb14 = t->ljb14.empty() ? nullptr : t->ljb14.data();
  s.excl_bounds = t->excl_bounds.data();
  s.excl_list = t->excl_list.data();
  s.pb_radii = t->pb_radii.data();
  s.gb_screen = t->gb_screen.data();
  s.gb_alpha = (t->igb >= 0) ? t->gb_alpha.data() : nullptr;
  s.gb_beta = (t->igb >= 0) ? t->gb_beta.data() : nullptr;
  s.gb_gamma = (t->igb >= 0) ? t->gb_gamma.data() : nullptr;
  s.nbond = static_cast<int>(t->bond_keq.size());
  s.bond_atoms = t->bond_atoms.data();
  s.bond_keq = t->bond_keq.data();
  s.bond_leq = t->bond_leq.data();
  s.nangl = static_cast<int>(t->angl_keq.size());
  s.angl_atoms = t->angl_atoms.data();
  s.angl_keq = t->angl_keq.data();
  s.angl_theta0 = t->angl_theta0.data();
  s.ndihe = static_cast<int>(t->dihe_amp.size());
  s.dihe_atoms = t->dihe_atoms.data();
  s.dihe_amp = t->dihe_amp.data();
  s.dihe_freq = t->dihe_freq.data();
  s.dihe_phase = t->dihe_phase.data();
  s.dihe_scee = t->dihe_scee.data();
  s.dihe_scnb = t->dihe_scnb.data();
  s.dihe_improper = t->dihe_improper.data();
  s.nubrd = static_cast<int>(t->ubrd_keq.size());
  s.ubrd_atoms = t->ubrd_atoms.empty() ? nullptr : t->ubrd_atoms.data();
  s.ubrd_keq = t->ubrd_keq.empty() ? nullptr : t->ubrd_keq.data();
  s.ubrd_leq = t->ubrd_leq.empty() ? nullptr : t->ubrd_leq.data();
  s.ncimp = static_cast<int>(t->cimp_keq.size());
  s.cimp_atoms = t->cimp_atoms.empty() ? nullptr : t->cimp_atoms.data();
  s.cimp_keq = t->cimp_keq.empty() ? nullptr : t->cimp_keq.data();
  s.cimp_phase = t->cimp_phase.empty() ? nullptr : t->cimp_phase.data();
  s.ncmap = static_cast<int>(t->cmap_surface.size());
  s.cmap_atoms = t->cmap_atoms.empty() ? nullptr : t->cmap_atoms.data();
  s.cmap_surface = t->cmap_surface.empty() ? nullptr : t->cmap_surface.data();
  s.ncmap_surf = (s.ncmap > 0) ? static_cast<int>(t->cmap_dims.size()) : 0;
  s.cmap_dims = (s.ncmap > 0) ? t->cmap_dims.data() : nullptr;
  s.cmap_values = (s.ncmap > 0) ? t->cmap_values.data() : nullptr;
  v->atomic_numbers = t->z_numbers.data();
  v->masses = t->mass.data();
  for (int lv = 0; lv < 3; lv++) {
    v->exclusion_bounds[lv] = t->nb_bounds[lv].data();
    v->exclusion_list[lv] = t->nb_list[lv].data();
  }
  v->radius_set = t->radius_set.c_str();
  v->title = t->title.c_str();
  v->implicit_solvent = t->igb;
  v->cmap_count = t->cmap_count;
  v->urey_bradley_count = t->urey_bradley_count;
  v->charmm_improper_count = t->charmm_improper_count;
  v->unit_cell = t->ifbox;
}

// ASCII restart / inpcrd: title, "natom [time]", then 3 natom coordinates in 12-column fields
// (six to a line); velocities and the box, when present, follow and are not read
void readCoordinates(const std::string &path, int natom, double* xyz) {
  std::ifstream in(path);
  if (!in) {
    throw Error(SB_ERR_ARGUMENT, "cannot open coordinate file " + path);
  }
  std::string line;
  if (!std::getline(in, line) || !std::getline(in, line)) {
    throw Error(SB_ERR_ARGUMENT, path + " is too short for an Amber coordinate file");
  }
  int nfile = 0;
  {
    std::istringstream ss(line);
    if (!(ss >> nfile) || nfile <= 0) {
      throw Error(SB_ERR_ARGUMENT, path + ": no atom count on the second line");
    }
  }
  if (nfile != natom) {
    throw Error(SB_ERR_ARGUMENT, path + " holds " + std::to_string(nfile) + " atoms, " +
                std::to_string(natom) + " expected");
  }
  const size_t want = 3 * static_cast<size_t>(natom);
  size_t got = 0;
  while (got < want && std::getline(in, line)) {
    line = trimRight(line);
    for (size_t p = 0; p < line.size() && got < want; p += 12) {
      const std::string f = line.substr(p, 12);
      const size_t a = f.find_first_not_of(' ');
      if (a == std::string::npos) {
        continue;
      }
      char* end = nullptr;
      const double v = std::strtod(f.c_str() + a, &end);
      if (end == f.c_str() + a || !std::isfinite(v)) {
        throw Error(SB_ERR_ARGUMENT, path + ": unreadable coordinate '" + f + "'");
      }
      xyz[got++] = v;
    }
  }
  if (got < want) {
    throw Error(SB_ERR_ARGUMENT, path + " ends after " + std::to_string(got) + " of " +
                std::to_string(want) + " coordinates");
  }
}

template <typename F> int hostGuarded(F &&f) {
  try {
    f();
    return SB_OK;
  }
  catch (const Error &e) {
    setLastError(e.what());
    return e.code;
  }
  catch (const std::exception &e) {
    setLastError(e.what());
    return SB_ERR_ARGUMENT;
  }
}

}  // namespace
}  // namespace sb

extern "C" int sb_read_amber_topology(const char* prmtop_path, sb_amber_topology** out) {
  return sb::hostGuarded([&]() {
    if (prmtop_path == nullptr || out == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "a file name and an output handle are required");
    }
    *out = nullptr;
    *out = sb::readTopology(prmtop_path);
  });
}

extern "C" int sb_amber_topology_view(const sb_amber_topology* top, sb_amber_view* view) {
  return sb::hostGuarded([&]() {
    if (top == nullptr || view == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "a topology handle and a view are required");
    }
    sb::fillView(top, view);
  });
}

extern "C" int sb_amber_set_implicit_solvent(sb_amber_topology* top, int igb, int radius_set) {
  return sb::hostGuarded([&]() {
    if (top == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "a topology handle is required");
    }
    sb::setImplicitSolvent(top, igb, radius_set);
  });
}

extern "C" int sb_amber_topology_destroy(sb_amber_topology* top) {
  delete top;
  return SB_OK;
}

extern "C" int sb_read_amber_coordinates(const char* inpcrd_path, int natom, double* xyz) {
  return sb::hostGuarded([&]() {
    if (inpcrd_path == nullptr || xyz == nullptr || natom <= 0) {
      throw sb::Error(SB_ERR_ARGUMENT, "a file name, an atom count and an output array are "
                      "required");
    }
    sb::readCoordinates(inpcrd_path, natom, xyz);
  });
}

extern "C" int sb_write_amber_coordinates(const char* inpcrd_path, const char* title, int natom,
                                          const double* xyz) {
  return sb::hostGuarded([&]() {
    if (inpcrd_path == nullptr || xyz == nullptr || natom <= 0 || natom > 9999999) {
      throw sb::Error(SB_ERR_ARGUMENT, "a file name, 1 to 9,999,999 atoms and their coordinates "
                      "are required");
    }
    const size_t n = 3 * static_cast<size_t>(natom);
    for (size_t k = 0; k < n; k++) {
      // %12.7f keeps a value in its field below 1e4 in magnitude
      if (!std::isfinite(xyz[k]) || std::fabs(xyz[k]) >= 9999.99999995) {
        throw sb::Error(SB_ERR_ARGUMENT, "coordinates must be finite and below 1e4 A in "
                        "magnitude to fit the Amber %12.7f fields");
      }
    }
    std::string text = (title != nullptr) ? title : "";
    if (text.find('\n') != std::string::npos) {
      throw sb::Error(SB_ERR_ARGUMENT, "the title must be one line");
    }
    text += '\n';
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%7d\n", natom);
    text += buf;
    for (size_t k = 0; k < n; k++) {
      std::snprintf(buf, sizeof(buf), "%12.7f", xyz[k]);
      // a value that rounds to zero prints unsigned, as STORMM's number formatting does
      // (Parsing/ascii_numbers.cpp:10-420)
      char* minus = std::strchr(buf, '-');
      if (minus != nullptr && std::strtod(buf, nullptr) == 0.0) {
        *minus = ' ';
      }
      text += buf;
      if (k % 6 == 5 || k + 1 == n) {
        text += '\n';
      }
    }
    std::ofstream out(inpcrd_path, std::ios::trunc);
    if (!out || !(out << text)) {
      throw sb::Error(SB_ERR_ARGUMENT, std::string("cannot write ") + inpcrd_path);
    }
  });
}
