// MDL MOL / SD file intake and output: the structures a conformer-minimization caller reads its
// molecules' coordinates from and writes its minimized conformers to.
//
// Reading follows STORMM's MdlMol for the V2000 format (MoleculeFormat/mdlmol.cpp:47-324,
// molecule_file_io.cpp:15-119): an SD file is split into compounds at "$$$$" lines (text of at
// least four lines before a marker makes a compound); a compound's MOL section ends at "M  END";
// the counts line gives the atom and bond counts (columns 1-3 and 4-6); atom lines give x, y, z
// in columns 1-30 (10 characters each), the element symbol in columns 32-34 and a charge code
// in 37-39 (1, 2, 3 -> +3, +2, +1; 5, 6, 7 -> -1, -2, -3; 4 = doublet radical, no charge);
// bond lines give the two 1-based atoms and the bond order (columns 1-3, 4-6, 7-9); "M  CHG"
// properties replace every atom-block charge of the compound (all atoms reset to zero, then the
// listed ones set); data items ("> <name>" followed by lines up to a blank line) keep their name
// and lines.  V3000 compounds are refused: STORMM's reader leaves them without atoms.
//
// Writing produces V2000 compounds that this reader, and STORMM's, read back to the same atoms,
// bonds, charges and data items, with coordinates in STORMM's %10.4f atom-line format.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "stormm_b200.h"
#include "synthesis.h"

namespace {

// Element symbols by atomic number (index 0 unused): IUPAC names, the table STORMM's
// symbolToZNumber maps against
const char* const kElements[] = {
  "",   "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",
  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga",
  "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag",
  "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu",
  "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au",
  "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U",  "Np", "Pu", "Am",
  "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds", "Rg",
  "Cn", "Nh", "Fl", "Mc", "Lv", "Ts", "Og"};
constexpr int kElementCount = sizeof(kElements) / sizeof(kElements[0]);

struct DataItem {
  std::string name;
  std::string content;     // lines joined by '\n'
};

struct Compound {
  std::string title, software, comment;
  std::vector<double> xyz;
  std::vector<int> znum, charge;
  std::vector<char> symbols;          // 4 characters per atom, NUL padded
  std::vector<int> bond_i, bond_j, bond_order;
  std::vector<DataItem> items;
  std::vector<const char*> item_names, item_contents;   // views for sb_sdf_compound
};

std::string trimmed(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) a++;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) b--;
  return s.substr(a, b - a);
}

// Columns [start, start + width) of a line, or "" past its end
std::string field(const std::string &line, size_t start, size_t width) {
  if (start >= line.size()) return std::string();
  return line.substr(start, std::min(width, line.size() - start));
}

bool hasInteger(const std::string &line, size_t start, size_t width) {
  const std::string f = trimmed(field(line, start, width));
  if (f.empty()) return false;
  size_t k = (f[0] == '-' || f[0] == '+') ? 1 : 0;
  if (k == f.size()) return false;
  for (; k < f.size(); k++) {
    if (f[k] < '0' || f[k] > '9') return false;
  }
  return true;
}

int integerField(const std::string &line, size_t start, size_t width, const std::string &what) {
  if (!hasInteger(line, start, width)) {
    throw sb::Error(SB_ERR_ARGUMENT, "SD file: " + what + " is not an integer: \"" +
                    field(line, start, width) + "\"");
  }
  return std::stoi(trimmed(field(line, start, width)));
}

double realField(const std::string &line, size_t start, size_t width, const std::string &what) {
  const std::string f = trimmed(field(line, start, width));
  char* end = nullptr;
  const double v = std::strtod(f.c_str(), &end);
  if (f.empty() || end == f.c_str() || *end != '\0' || !std::isfinite(v)) {
    throw sb::Error(SB_ERR_ARGUMENT, "SD file: " + what + " is not a number: \"" + f + "\"");
  }
  return v;
}

int atomicNumber(const std::string &sym) {
  for (int z = 1; z < kElementCount; z++) {
    if (sym == kElements[z]) return z;
  }
  return 0;   // not an element (query atoms, pseudo-atoms)
}

bool startsWith(const std::string &line, const char* tag) {
  return line.compare(0, std::strlen(tag), tag) == 0;
}

// One compound from lines [begin, end) of the file
Compound parseCompound(const std::vector<std::string> &lines, size_t begin, size_t end,
                       size_t index) {
  const std::string where = "SD file compound " + std::to_string(index);
  Compound c;
  c.title = trimmed(lines[begin]);
  c.software = trimmed(lines[begin + 1]);
  c.comment = trimmed(lines[begin + 2]);
  const std::string &counts = lines[begin + 3];
  if (counts.find("V3000") != std::string::npos || counts.find("v3000") != std::string::npos) {
    throw sb::Error(SB_ERR_UNSUPPORTED, where + " is in the V3000 format; only V2000 is read");
  }
  if (counts.find("V2000") == std::string::npos && counts.find("v2000") == std::string::npos) {
    throw sb::Error(SB_ERR_ARGUMENT, where + " has no V2000 counts line");
  }
  const int natom = integerField(counts, 0, 3, where + " atom count");
  const int nbond = integerField(counts, 3, 3, where + " bond count");
  if (natom <= 0 || nbond < 0) {
    throw sb::Error(SB_ERR_ARGUMENT, where + " lists " + std::to_string(natom) + " atoms and " +
                    std::to_string(nbond) + " bonds");
  }
  size_t mol_end = begin;
  while (mol_end < end && !startsWith(lines[mol_end], "M  END")) mol_end++;
  if (begin + 4 + static_cast<size_t>(natom) + static_cast<size_t>(nbond) > mol_end) {
    throw sb::Error(SB_ERR_ARGUMENT, where + " ends before its atom and bond blocks do");
  }
  c.xyz.resize(3 * static_cast<size_t>(natom));
  c.znum.resize(natom);
  c.charge.assign(natom, 0);
  c.symbols.assign(4 * static_cast<size_t>(natom), '\0');
  for (int a = 0; a < natom; a++) {
    const std::string &ln = lines[begin + 4 + a];
    const std::string what = where + " atom " + std::to_string(a + 1);
    c.xyz[3 * a] = realField(ln, 0, 10, what + " x");
    c.xyz[3 * a + 1] = realField(ln, 10, 10, what + " y");
    c.xyz[3 * a + 2] = realField(ln, 20, 10, what + " z");
    const std::string sym = trimmed(field(ln, 31, 3));
    std::memcpy(&c.symbols[4 * static_cast<size_t>(a)], sym.data(), std::min<size_t>(3, sym.size()));
    c.znum[a] = atomicNumber(sym);
    if (hasInteger(ln, 36, 3)) {
      const int code = integerField(ln, 36, 3, what + " charge code");
      static const int kCodeCharge[8] = {0, 3, 2, 1, 0, -1, -2, -3};
      if (code < 0 || code > 7) {
        throw sb::Error(SB_ERR_ARGUMENT, what + ": charge code " + std::to_string(code) +
                        " is not an MDL code (0-7)");
      }
      c.charge[a] = kCodeCharge[code];
    }
  }
  for (int b = 0; b < nbond; b++) {
    const std::string &ln = lines[begin + 4 + natom + b];
    const std::string what = where + " bond " + std::to_string(b + 1);
    const int i = integerField(ln, 0, 3, what + " first atom") - 1;
    const int j = integerField(ln, 3, 3, what + " second atom") - 1;
    if (i < 0 || i >= natom || j < 0 || j >= natom) {
      throw sb::Error(SB_ERR_ARGUMENT, what + " names an atom outside the compound");
    }
    const int order = hasInteger(ln, 6, 3) ? integerField(ln, 6, 3, what + " order") : 1;
    if (order < 1 || order > 8) {
      throw sb::Error(SB_ERR_ARGUMENT, what + ": bond type " + std::to_string(order) +
                      " is not an MDL type (1-8)");
    }
    c.bond_i.push_back(i);
    c.bond_j.push_back(j);
    c.bond_order.push_back(order);
  }
  // properties: "M  CHG" replaces all atom-block charges
  bool reset = false;
  for (size_t l = begin + 4 + natom + nbond; l < mol_end; l++) {
    const std::string &ln = lines[l];
    if (!startsWith(ln, "M  CHG")) continue;
    if (!reset) {
      std::fill(c.charge.begin(), c.charge.end(), 0);
      reset = true;
    }
    const int n = integerField(ln, 6, 3, where + " M  CHG entry count");
    for (int e = 0; e < n; e++) {
      const int a = integerField(ln, 10 + 8 * e, 3, where + " M  CHG atom") - 1;
      const int q = integerField(ln, 14 + 8 * e, 3, where + " M  CHG charge");
      if (a < 0 || a >= natom) {
        throw sb::Error(SB_ERR_ARGUMENT, where + ": M  CHG names an atom outside the compound");
      }
      c.charge[a] = q;
    }
  }
  // data items after the MOL section
  for (size_t l = mol_end + 1; l < end; l++) {
    const std::string &ln = lines[l];
    if (ln.empty() || ln[0] != '>') continue;
    DataItem it;
    const size_t lt = ln.find('<');
    const size_t gt = (lt == std::string::npos) ? lt : ln.find('>', lt);
    if (lt != std::string::npos && gt != std::string::npos) {
      it.name = ln.substr(lt + 1, gt - lt - 1);
    }
    size_t k = l + 1;
    for (; k < end && !trimmed(lines[k]).empty(); k++) {
      if (!it.content.empty()) it.content += '\n';
      it.content += lines[k];
    }
    c.items.push_back(std::move(it));
    l = k;
  }
  for (const DataItem &it : c.items) {
    c.item_names.push_back(it.name.c_str());
    c.item_contents.push_back(it.content.c_str());
  }
  return c;
}

std::vector<Compound> readSdf(const std::string &path) {
  std::ifstream in(path);
  if (!in) {
    throw sb::Error(SB_ERR_ARGUMENT, "cannot open SD file " + path);
  }
  std::vector<std::string> lines;
  std::string ln;
  while (std::getline(in, ln)) {
    if (!ln.empty() && ln.back() == '\r') ln.pop_back();
    lines.push_back(ln);
  }
  // compounds: text of four or more lines before each "$$$$", and after the last one
  std::vector<std::pair<size_t, size_t>> spans;
  size_t start = 0;
  for (size_t l = 0; l < lines.size(); l++) {
    if (startsWith(lines[l], "$$$$")) {
      if (l - start >= 4) spans.emplace_back(start, l);
      start = l + 1;
    }
  }
  if (lines.size() >= start + 4) spans.emplace_back(start, lines.size());
  if (spans.empty()) {
    throw sb::Error(SB_ERR_ARGUMENT, "SD file " + path + " holds no compound");
  }
  std::vector<Compound> out;
  for (size_t k = 0; k < spans.size(); k++) {
    out.push_back(parseCompound(lines, spans[k].first, spans[k].second, k));
  }
  return out;
}

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

struct sb_sdf {
  std::vector<Compound> compounds;
};

extern "C" {

int sb_read_sdf(const char* path, sb_sdf** out) {
  return guarded([&]() {
    if (path == nullptr || out == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_read_sdf: null argument");
    }
    *out = nullptr;
    auto h = std::make_unique<sb_sdf>();
    h->compounds = readSdf(path);
    *out = h.release();
  });
}

int sb_sdf_compound_count(const sb_sdf* sdf, int* count) {
  return guarded([&]() {
    if (sdf == nullptr || count == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_sdf_compound_count: null argument");
    }
    *count = static_cast<int>(sdf->compounds.size());
  });
}

int sb_sdf_compound(const sb_sdf* sdf, int index, sb_sdf_view* view) {
  return guarded([&]() {
    if (sdf == nullptr || view == nullptr) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_sdf_compound: null argument");
    }
    if (index < 0 || index >= static_cast<int>(sdf->compounds.size())) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_sdf_compound: index out of range");
    }
    const Compound &c = sdf->compounds[index];
    std::memset(view, 0, sizeof(sb_sdf_view));
    view->title = c.title.c_str();
    view->natom = static_cast<int>(c.znum.size());
    view->xyz = c.xyz.data();
    view->atomic_number = c.znum.data();
    view->formal_charge = c.charge.data();
    view->symbols = c.symbols.data();
    view->nbond = static_cast<int>(c.bond_i.size());
    view->bond_i = c.bond_i.empty() ? nullptr : c.bond_i.data();
    view->bond_j = c.bond_j.empty() ? nullptr : c.bond_j.data();
    view->bond_order = c.bond_order.empty() ? nullptr : c.bond_order.data();
    view->n_items = static_cast<int>(c.items.size());
    view->item_names = c.item_names.empty() ? nullptr : c.item_names.data();
    view->item_contents = c.item_contents.empty() ? nullptr : c.item_contents.data();
  });
}

int sb_sdf_destroy(sb_sdf* sdf) {
  delete sdf;
  return SB_OK;
}

int sb_write_sdf_compound(const char* path, int append, const sb_sdf_view* c) {
  return guarded([&]() {
    if (path == nullptr || c == nullptr || c->natom <= 0 || c->natom > 999 || c->nbond < 0 ||
        c->nbond > 999 || c->xyz == nullptr ||
        (c->symbols == nullptr && c->atomic_number == nullptr) ||
        (c->nbond > 0 && (c->bond_i == nullptr || c->bond_j == nullptr)) ||
        (c->n_items > 0 && (c->item_names == nullptr || c->item_contents == nullptr))) {
      throw sb::Error(SB_ERR_ARGUMENT, "sb_write_sdf_compound: a compound needs 1-999 atoms, "
                      "at most 999 bonds, coordinates, symbols or atomic numbers and its bond "
                      "and data-item arrays");
    }
    std::ostringstream os;
    char buf[128];
    os << (c->title ? c->title : "") << "\n  stormm_b200\n\n";
    std::snprintf(buf, sizeof(buf), "%3d%3d  0  0  0  0  0  0  0  0999 V2000\n", c->natom,
                  c->nbond);
    os << buf;
    std::vector<std::pair<int, int>> charged;
    for (int a = 0; a < c->natom; a++) {
      std::string sym;
      if (c->symbols != nullptr) {
        sym.assign(c->symbols + 4 * static_cast<size_t>(a),
                   strnlen(c->symbols + 4 * static_cast<size_t>(a), 3));
      }
      else {
        const int z = c->atomic_number[a];
        if (z < 1 || z >= kElementCount) {
          throw sb::Error(SB_ERR_ARGUMENT, "sb_write_sdf_compound: atomic number out of range");
        }
        sym = kElements[z];
      }
      const double x = c->xyz[3 * a], y = c->xyz[3 * a + 1], z = c->xyz[3 * a + 2];
      if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z) || std::fabs(x) >= 1e5 ||
          std::fabs(y) >= 1e5 || std::fabs(z) >= 1e5) {
        throw sb::Error(SB_ERR_ARGUMENT, "sb_write_sdf_compound: coordinates must be finite "
                        "and fit the %10.4f atom-line fields");
      }
      std::snprintf(buf, sizeof(buf), "%10.4f%10.4f%10.4f %-3s 0  0  0  0  0  0  0  0  0  0  0  0\n",
                    x, y, z, sym.c_str());
      os << buf;
      const int q = (c->formal_charge != nullptr) ? c->formal_charge[a] : 0;
      if (q != 0) charged.emplace_back(a + 1, q);
    }
    for (int b = 0; b < c->nbond; b++) {
      const int order = (c->bond_order != nullptr) ? c->bond_order[b] : 1;
      if (c->bond_i[b] < 0 || c->bond_i[b] >= c->natom || c->bond_j[b] < 0 ||
          c->bond_j[b] >= c->natom || order < 1 || order > 8) {
        throw sb::Error(SB_ERR_ARGUMENT, "sb_write_sdf_compound: bond atom or type out of range");
      }
      std::snprintf(buf, sizeof(buf), "%3d%3d%3d  0\n", c->bond_i[b] + 1, c->bond_j[b] + 1, order);
      os << buf;
    }
    // charges as "M  CHG" properties, at most eight per line
    for (size_t k = 0; k < charged.size(); k += 8) {
      const size_t n = std::min<size_t>(8, charged.size() - k);
      std::snprintf(buf, sizeof(buf), "M  CHG%3zu", n);
      os << buf;
      for (size_t e = 0; e < n; e++) {
        std::snprintf(buf, sizeof(buf), " %3d %3d", charged[k + e].first, charged[k + e].second);
        os << buf;
      }
      os << "\n";
    }
    os << "M  END\n";
    for (int it = 0; it < c->n_items; it++) {
      os << "> <" << (c->item_names[it] ? c->item_names[it] : "") << ">\n"
         << (c->item_contents[it] ? c->item_contents[it] : "") << "\n\n";
    }
    os << "$$$$\n";
    std::ofstream out(path, append ? std::ios::app : std::ios::trunc);
    if (!out) {
      throw sb::Error(SB_ERR_ARGUMENT, std::string("cannot write SD file ") + path);
    }
    out << os.str();
  });
}

}  // extern "C"
