// Seeded synthetic molecule builder for the batched implicit-solvent workloads.
//
// Builds a random tree of heavy atoms (or a polymer-like chain) in 3-D with clash rejection,
// fills free valences with hydrogens, and parameterises bonds, angles, dihedrals, charges,
// Lennard-Jones types and GB radii.  Every real-valued parameter is rounded to nine significant
// digits and every charge to a multiple of 2^-23 e, so that an Amber prmtop written from the
// molecule is read back by STORMM's AtomGraph (Topology/atomgraph_detailers.cpp:800-1115; charge
// smoothing Topology/atomgraph_refinement.cpp:1519) to exactly the same numbers.
//
// This is workload-generation code for tests and benchmarks.  It is compiled into its own small
// library (libstormm_b200_synth.so) and exposes a C ABI used through ctypes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTheta0 = 109.5 * kPi / 180.0;
constexpr double kChargeQuantum = 1.0 / 8388608.0;

// xoshiro256** seeded through splitmix64
class Rng {
public:
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) {
      x += 0x9e3779b97f4a7c15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s_[i] = z ^ (z >> 31);
    }
  }
  uint64_t next() {
    const uint64_t result = rotl(s_[1] * 5, 7) * 9;
    const uint64_t t = s_[1] << 17;
    s_[2] ^= s_[0];
    s_[3] ^= s_[1];
    s_[1] ^= s_[2];
    s_[0] ^= s_[3];
    s_[2] ^= t;
    s_[3] = rotl(s_[3], 45);
    return result;
  }
  double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double lo, double hi) { return lo + (hi - lo) * uniform(); }
  int integer(int lo, int hi_exclusive) {
    return lo + static_cast<int>(uniform() * (hi_exclusive - lo));
  }
  double normal() {
    // Box-Muller, one value per call
    double u1 = uniform();
    while (u1 <= 1.0e-300) {
      u1 = uniform();
    }
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
  }
private:
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t s_[4];
};

struct V3 {
  double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double norm(V3 a) { return std::sqrt(dot(a, a)); }
V3 unit(V3 a) {
  const double n = norm(a);
  return (n > 1.0e-12) ? (1.0 / n) * a : V3{1.0, 0.0, 0.0};
}
V3 randomUnit(Rng &rng) { return unit({rng.normal(), rng.normal(), rng.normal()}); }

double sig9(double v) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.8E", v);
  return std::strtod(buf, nullptr);
}
double round_to(double v, int decimals) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.*f", decimals, v);
  return std::strtod(buf, nullptr);
}

// Candidate unit vectors for a new bond, roughly tetrahedral to the existing bonds
std::vector<V3> candidates(Rng &rng, const std::vector<V3> &dirs, int count) {
  std::vector<V3> out;
  const size_t m = dirs.size();
  if (m == 0) {
    for (int k = 0; k < count; k++) {
      out.push_back(randomUnit(rng));
    }
  }
  else if (m == 1) {
    const V3 b = dirs[0];
    V3 perp = unit(cross(b, randomUnit(rng)));
    const V3 perp2 = cross(b, perp);
    const double c = std::cos(kTheta0), s = std::sin(kTheta0);
    for (int k = 0; k < count; k++) {
      const double phi = 2.0 * kPi * (k + rng.uniform()) / count;
      out.push_back(c * b + s * (std::cos(phi) * perp + std::sin(phi) * perp2));
    }
  }
  else if (m == 2) {
    V3 bis = (-1.0) * (dirs[0] + dirs[1]);
    bis = (norm(bis) > 1.0e-6) ? unit(bis) : randomUnit(rng);
    V3 n = cross(dirs[0], dirs[1]);
    n = (norm(n) > 1.0e-6) ? unit(n) : randomUnit(rng);
    const double half = 54.75 * kPi / 180.0;
    out.push_back(std::cos(half) * bis + std::sin(half) * n);
    out.push_back(std::cos(half) * bis - std::sin(half) * n);
  }
  else {
    V3 d = {0.0, 0.0, 0.0};
    for (const V3 &b : dirs) {
      d = d - b;
    }
    out.push_back((norm(d) > 1.0e-6) ? unit(d) : randomUnit(rng));
  }
  for (V3 &d : out) {
    d = unit(d + V3{0.05 * rng.normal(), 0.05 * rng.normal(), 0.05 * rng.normal()});
  }
  // Keep only directions whose angle to every existing bond lies in [85, 130] degrees, topping
  // up with random directions in that window: near-linear bond angles make the dihedrals through
  // them singular.
  auto in_window = [&](const V3 &d) {
    for (const V3 &b : dirs) {
      const double c = dot(d, b);
      if (c > std::cos(85.0 * kPi / 180.0) || c < std::cos(130.0 * kPi / 180.0)) {
        return false;
      }
    }
    return true;
  };
  std::vector<V3> kept;
  for (const V3 &d : out) {
    if (in_window(d)) kept.push_back(d);
  }
  for (int t = 0; t < 200 && static_cast<int>(kept.size()) < std::max(count / 2, 2); t++) {
    const V3 d = randomUnit(rng);
    if (in_window(d)) kept.push_back(d);
  }
  if (kept.empty()) {
    kept = out;
  }
  return kept;
}

// Uniform cell grid for clash checks
class Grid {
public:
  explicit Grid(double cell) : cell_(cell) {}
  void add(int a, V3 p) { cells_[key(p)].push_back(a); }
  // minimum distance from p to any atom in the grid except those in skip (within reach)
  double minDistance(V3 p, const std::vector<V3> &pos, const std::vector<int> &skip,
                     double reach) const {
    double best2 = reach * reach;
    const long kx = fl(p.x), ky = fl(p.y), kz = fl(p.z);
    for (long dx = -1; dx <= 1; dx++) {
      for (long dy = -1; dy <= 1; dy++) {
        for (long dz = -1; dz <= 1; dz++) {
          auto it = cells_.find(pack(kx + dx, ky + dy, kz + dz));
          if (it == cells_.end()) {
            continue;
          }
          for (int a : it->second) {
            if (std::find(skip.begin(), skip.end(), a) != skip.end()) {
              continue;
            }
            const V3 d = pos[a] - p;
            best2 = std::min(best2, dot(d, d));
          }
        }
      }
    }
    return std::sqrt(best2);
  }
private:
  long fl(double v) const { return static_cast<long>(std::floor(v / cell_)); }
  static uint64_t pack(long x, long y, long z) {
    return (static_cast<uint64_t>(x & 0x1fffff) << 42) | (static_cast<uint64_t>(y & 0x1fffff) << 21) |
           static_cast<uint64_t>(z & 0x1fffff);
  }
  uint64_t key(V3 p) const { return pack(fl(p.x), fl(p.y), fl(p.z)); }
  double cell_;
  struct Hash {
    size_t operator()(uint64_t k) const { return std::hash<uint64_t>()(k * 0x9e3779b97f4a7c15ULL); }
  };
  std::unordered_map<uint64_t, std::vector<int>, Hash> cells_;
};

}  // namespace

extern "C" {

// A molecule as flat arrays (0-based indices).  All arrays are owned by the library and released
// with sbsyn_free().
typedef struct {
  int natom, nbond, nangl, ndihe, ntype;
  double* coords;       // natom * 3
  double* charge;       // natom
  int* lj_idx;          // natom
  double* lja;          // ntype * ntype
  double* ljb;          // ntype * ntype
  int* z_numbers;       // natom
  double* mass;         // natom
  double* pb_radii;     // natom
  double* gb_screen;    // natom
  int* bonds;           // nbond * 2
  double* bond_k;
  double* bond_r0;
  int* angles;          // nangl * 3
  double* angl_k;
  double* angl_theta0;
  int* dihedrals;       // ndihe * 4
  double* dihe_amp;
  double* dihe_freq;
  double* dihe_phase;
  int* dihe_has14;      // ndihe, 1 if the term carries the I-L 1-4 pair
} sbsyn_molecule;

void sbsyn_free(sbsyn_molecule* m);
int sbsyn_make_molecule(uint64_t seed, int natom, double noise, int kind, sbsyn_molecule* out);

}  // extern "C"

namespace {

template <typename T> T* copyOut(const std::vector<T> &v) {
  T* p = static_cast<T*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
  if (!v.empty()) {
    std::memcpy(p, v.data(), v.size() * sizeof(T));
  }
  return p;
}

struct Builder {
  Rng rng;
  int natom;
  std::vector<V3> pos;
  std::vector<int> z, parent, used, capv;
  std::vector<double> blen;
  std::vector<std::vector<V3>> dirs;
  std::vector<std::vector<int>> nbrs;
  Grid grid{3.0};

  Builder(uint64_t seed, int n) : rng(seed), natom(n) {
    pos.reserve(n);
  }

  int commit(int par, V3 p, double r, int zz, int cv) {
    const int a = pos.size();
    pos.push_back(p);
    z.push_back(zz);
    capv.push_back(cv);
    used.push_back(0);
    parent.push_back(par);
    blen.push_back(r);
    dirs.emplace_back();
    nbrs.emplace_back();
    if (par >= 0) {
      const V3 d = (1.0 / r) * (p - pos[par]);
      dirs[par].push_back(d);
      dirs[a].push_back((-1.0) * d);
      nbrs[par].push_back(a);
      nbrs[a].push_back(par);
      used[par]++;
      used[a]++;
    }
    grid.add(a, p);
    return a;
  }

  // best candidate position around parent par; returns the minimum distance achieved
  double tryPlace(int par, double r, double clash, V3 *out) {
    std::vector<int> skip = nbrs[par];
    skip.push_back(par);
    const std::vector<V3> cands = candidates(rng, dirs[par], 12);
    double best_d = -1.0;
    for (const V3 &d : cands) {
      const V3 p = pos[par] + r * d;
      const double dmin = grid.minDistance(p, pos, skip, 3.0);
      if (dmin > best_d) {
        best_d = dmin;
        *out = p;
      }
      if (dmin >= clash) {
        break;
      }
    }
    return best_d;
  }
};

void parameterise(Rng &rng, int natom, const std::vector<V3> &coords, const std::vector<int> &z,
                  const std::vector<std::pair<int, int>> &bonds, const std::vector<double> &r0,
                  double noise, double theta0, bool second_terms, sbsyn_molecule* out) {
  std::vector<std::vector<int>> nbr(natom);
  for (const auto &b : bonds) {
    nbr[b.first].push_back(b.second);
    nbr[b.second].push_back(b.first);
  }
  for (auto &v : nbr) {
    std::sort(v.begin(), v.end());
  }
  // angles
  std::vector<int> angl;
  for (int j = 0; j < natom; j++) {
    for (size_t a = 0; a < nbr[j].size(); a++) {
      for (size_t b = a + 1; b < nbr[j].size(); b++) {
        angl.push_back(nbr[j][a]);
        angl.push_back(j);
        angl.push_back(nbr[j][b]);
      }
    }
  }
  // dihedrals
  std::vector<int> dihe, has14;
  std::vector<double> amp, freq, phase;
  for (const auto &b : bonds) {
    const int j = b.first, k = b.second;
    for (int i : nbr[j]) {
      if (i == k) continue;
      for (int l : nbr[k]) {
        if (l == j || l == i) continue;
        const int n1 = rng.integer(1, 4);
        dihe.insert(dihe.end(), {i, j, k, l});
        amp.push_back(round_to(rng.uniform(0.1, 2.0), 4));
        freq.push_back(n1);
        phase.push_back(sig9(rng.uniform() < 0.5 ? 0.0 : kPi));
        has14.push_back(1);
        if (second_terms && rng.uniform() < 0.25) {
          dihe.insert(dihe.end(), {i, j, k, l});
          amp.push_back(round_to(rng.uniform(0.1, 2.0), 4));
          freq.push_back(1 + (n1 % 3));
          phase.push_back(sig9(rng.uniform() < 0.5 ? 0.0 : kPi));
          has14.push_back(0);
        }
      }
    }
  }
  // charges: N(0, 0.3), net zero, multiples of 2^-23 with an exact integer sum of zero
  std::vector<double> q(natom);
  double qm = 0.0;
  for (int i = 0; i < natom; i++) {
    q[i] = 0.3 * rng.normal();
    qm += q[i];
  }
  qm /= natom;
  std::vector<long long> qi(natom);
  long long qsum = 0;
  int qmax = 0;
  for (int i = 0; i < natom; i++) {
    qi[i] = std::llround((q[i] - qm) / kChargeQuantum);
    qsum += qi[i];
    if (std::llabs(qi[i]) > std::llabs(qi[qmax])) qmax = i;
  }
  qi[qmax] -= qsum;
  for (int i = 0; i < natom; i++) {
    q[i] = static_cast<double>(qi[i]) * kChargeQuantum;
  }
  // Lennard-Jones types
  const int nt = 8;
  std::vector<double> sigma(nt), eps(nt);
  for (int t = 0; t < nt; t++) {
    sigma[t] = rng.uniform(2.0, 3.8);
    eps[t] = rng.uniform(0.02, 0.2);
  }
  std::sort(sigma.begin(), sigma.end());
  std::vector<double> lja(nt * nt), ljb(nt * nt);
  for (int a = 0; a < nt; a++) {
    for (int b = 0; b < nt; b++) {
      const double s = 0.5 * (sigma[a] + sigma[b]);
      const double e = std::sqrt(eps[a] * eps[b]);
      const double s6 = s * s * s * s * s * s;
      lja[a * nt + b] = sig9(4.0 * e * s6 * s6);
      ljb[a * nt + b] = sig9(4.0 * e * s6);
    }
  }
  std::vector<int> lj_idx(natom);
  std::vector<double> rad(natom), scr(natom), mass(natom), xyz(3 * natom);
  for (int i = 0; i < natom; i++) {
    lj_idx[i] = (z[i] == 1) ? rng.integer(0, 2) : rng.integer(2, nt);
    rad[i] = round_to((z[i] == 1) ? rng.uniform(1.2, 1.3) : rng.uniform(1.5, 1.9), 4);
    scr[i] = round_to(rng.uniform(0.72, 0.85), 4);
    mass[i] = (z[i] == 1) ? 1.008 : (z[i] == 6) ? 12.01 : (z[i] == 7) ? 14.01 : 16.0;
    xyz[3 * i] = round_to(coords[i].x + noise * rng.normal(), 7);
    xyz[3 * i + 1] = round_to(coords[i].y + noise * rng.normal(), 7);
    xyz[3 * i + 2] = round_to(coords[i].z + noise * rng.normal(), 7);
  }
  std::vector<int> bnd;
  std::vector<double> bk, br0;
  for (size_t t = 0; t < bonds.size(); t++) {
    bnd.push_back(bonds[t].first);
    bnd.push_back(bonds[t].second);
    bk.push_back(round_to(rng.uniform(300.0, 600.0), 2));
    br0.push_back(round_to(r0[t], 4));
  }
  std::vector<double> ak, ath;
  for (size_t t = 0; t < angl.size() / 3; t++) {
    ak.push_back(round_to(rng.uniform(50.0, 80.0), 2));
    ath.push_back(sig9(theta0));
  }
  out->natom = natom;
  out->nbond = bonds.size();
  out->nangl = angl.size() / 3;
  out->ndihe = dihe.size() / 4;
  out->ntype = nt;
  out->coords = copyOut(xyz);
  out->charge = copyOut(q);
  out->lj_idx = copyOut(lj_idx);
  out->lja = copyOut(lja);
  out->ljb = copyOut(ljb);
  out->z_numbers = copyOut(z);
  out->mass = copyOut(mass);
  out->pb_radii = copyOut(rad);
  out->gb_screen = copyOut(scr);
  out->bonds = copyOut(bnd);
  out->bond_k = copyOut(bk);
  out->bond_r0 = copyOut(br0);
  out->angles = copyOut(angl);
  out->angl_k = copyOut(ak);
  out->angl_theta0 = copyOut(ath);
  out->dihedrals = copyOut(dihe);
  out->dihe_amp = copyOut(amp);
  out->dihe_freq = copyOut(freq);
  out->dihe_phase = copyOut(phase);
  out->dihe_has14 = copyOut(has14);
}

int makeTree(uint64_t seed, int natom, double noise, sbsyn_molecule* out) {
  Builder bld(seed, natom);
  Rng &rng = bld.rng;
  const int n_heavy = std::max(1, static_cast<int>(std::lround(natom * 24.0 / 64.0)));
  const int n_h = natom - n_heavy;
  const int valence[3] = {4, 3, 2};
  const int znum[3] = {6, 7, 8};
  std::vector<int> ek(n_heavy);
  for (int k = 0; k < n_heavy; k++) {
    const int r = rng.integer(0, 6);
    ek[k] = (r < 4) ? 0 : (r == 4) ? 1 : 2;
  }
  auto capacity = [&]() {
    int c = 0;
    for (int e : ek) c += valence[e];
    return c - 2 * (n_heavy - 1);
  };
  while (capacity() < n_h) {
    int worst = 0;
    for (int k = 1; k < n_heavy; k++) {
      if (valence[ek[k]] < valence[ek[worst]]) worst = k;
    }
    if (ek[worst] == 0) return 1;
    ek[worst] = 0;
  }
  std::vector<int> heavy_ids;
  heavy_ids.push_back(bld.commit(-1, {0.0, 0.0, 0.0}, 0.0, znum[ek[0]], valence[ek[0]]));
  const double heavy_clash[5] = {2.7, 2.5, 2.3, 2.0, 1.8};
  for (int k = 1; k < n_heavy; k++) {
    bool placed = false;
    for (int pass = 0; pass < 5 && !placed; pass++) {
      const double clash = heavy_clash[pass];
      std::vector<int> open;
      for (int a : heavy_ids) {
        if (bld.used[a] < bld.capv[a]) open.push_back(a);
      }
      if (open.empty() || pass >= 3) {
        // widen the search to every heavy atom, opening one extra valence on the one used
        open = heavy_ids;
      }
      std::vector<int> pool = (pass < 2) ?
        std::vector<int>(open.end() - std::min<size_t>(4, open.size()), open.end()) : open;
      for (size_t t = pool.size(); t > 1; t--) {
        std::swap(pool[t - 1], pool[rng.integer(0, t)]);
      }
      for (int par : pool) {
        const double r = rng.uniform(1.40, 1.54);
        V3 p;
        if (bld.tryPlace(par, r, clash, &p) >= clash) {
          if (bld.used[par] >= bld.capv[par]) bld.capv[par]++;
          heavy_ids.push_back(bld.commit(par, p, r, znum[ek[k]], valence[ek[k]]));
          placed = true;
          break;
        }
      }
    }
    if (!placed) {
      const int par = heavy_ids.back();
      const double r = rng.uniform(1.40, 1.54);
      V3 p;
      bld.tryPlace(par, r, 0.0, &p);
      bld.capv[par]++;
      heavy_ids.push_back(bld.commit(par, p, r, znum[ek[k]], valence[ek[k]]));
    }
  }
  const double h_clash[4] = {2.2, 2.0, 1.8, 1.6};
  for (int h = 0; h < n_h; h++) {
    bool placed = false;
    for (double clash : h_clash) {
      std::vector<int> open;
      for (int a : heavy_ids) {
        if (bld.used[a] < bld.capv[a]) open.push_back(a);
      }
      for (size_t t = open.size(); t > 1; t--) {
        std::swap(open[t - 1], open[rng.integer(0, t)]);
      }
      for (int par : open) {
        const double r = rng.uniform(1.00, 1.10);
        V3 p;
        if (bld.tryPlace(par, r, clash, &p) >= clash) {
          bld.commit(par, p, r, 1, 1);
          placed = true;
          break;
        }
      }
      if (placed) break;
    }
    if (!placed) {
      // No open valence has room: take the roomiest spot next to any heavy atom, letting that
      // atom exceed its nominal valence.
      double best_d = -1.0;
      int best_par = heavy_ids[0];
      V3 best_p = {0.0, 0.0, 0.0};
      const double r = rng.uniform(1.00, 1.10);
      for (int par : heavy_ids) {
        for (int t = 0; t < 24; t++) {
          const V3 dir = randomUnit(rng);
          // keep every bond angle at the parent between 85 and 130 degrees
          bool ok = true;
          for (const V3 &b : bld.dirs[par]) {
            const double c = dot(dir, b);
            if (c > std::cos(85.0 * kPi / 180.0) || c < std::cos(130.0 * kPi / 180.0)) {
              ok = false;
              break;
            }
          }
          if (!ok) continue;
          const V3 p = bld.pos[par] + r * dir;
          std::vector<int> skip = bld.nbrs[par];
          skip.push_back(par);
          const double d = bld.grid.minDistance(p, bld.pos, skip, 3.0);
          if (d > best_d) {
            best_d = d;
            best_par = par;
            best_p = p;
          }
        }
      }
      if (best_d < 0.0) {
        best_p = bld.pos[best_par] + r * randomUnit(rng);
      }
      bld.capv[best_par]++;
      bld.commit(best_par, best_p, r, 1, 1);
    }
  }
  // atom order: each heavy atom followed by its hydrogens
  std::vector<int> new_index(natom, -1);
  int idx = 0;
  for (int hv : heavy_ids) {
    new_index[hv] = idx++;
    for (int a : bld.nbrs[hv]) {
      if (bld.z[a] == 1) new_index[a] = idx++;
    }
  }
  if (idx != natom) return 3;
  std::vector<V3> coords(natom);
  std::vector<int> z(natom);
  for (int a = 0; a < natom; a++) {
    coords[new_index[a]] = bld.pos[a];
    z[new_index[a]] = bld.z[a];
  }
  std::vector<std::pair<int, int>> bonds;
  std::vector<double> r0;
  std::vector<std::pair<long long, int>> order;
  for (int a = 0; a < natom; a++) {
    if (bld.parent[a] >= 0) {
      const int i = new_index[bld.parent[a]], j = new_index[a];
      bonds.push_back({std::min(i, j), std::max(i, j)});
      r0.push_back(bld.blen[a]);
    }
  }
  for (size_t t = 0; t < bonds.size(); t++) {
    order.push_back({static_cast<long long>(bonds[t].first) * natom + bonds[t].second,
                     static_cast<int>(t)});
  }
  std::sort(order.begin(), order.end());
  std::vector<std::pair<int, int>> sb;
  std::vector<double> sr;
  for (const auto &o : order) {
    sb.push_back(bonds[o.second]);
    sr.push_back(r0[o.second]);
  }
  parameterise(rng, natom, coords, z, sb, sr, noise, kTheta0, true, out);
  return 0;
}

int makeChain(uint64_t seed, int natom, double noise, sbsyn_molecule* out) {
  Builder bld(seed, natom);
  Rng &rng = bld.rng;
  bld.commit(-1, {0.0, 0.0, 0.0}, 0.0, 6, 4);
  V3 prev_dir = {1.0, 0.0, 0.0};
  for (int k = 1; k < natom; k++) {
    V3 best_p = bld.pos[k - 1] + 1.5 * prev_dir;
    double best_d = -1.0;
    V3 best_dir = prev_dir;
    for (int t = 0; t < 200; t++) {
      const V3 d = randomUnit(rng);
      const double c = dot(d, prev_dir);
      if (k > 1 && (c > std::cos(60.0 * kPi / 180.0) || c < std::cos(80.0 * kPi / 180.0))) {
        continue;
      }
      const V3 p = bld.pos[k - 1] + 1.5 * d;
      std::vector<int> skip = {k - 1};
      if (k >= 2) skip.push_back(k - 2);
      const double dmin = bld.grid.minDistance(p, bld.pos, skip, 3.0);
      if (dmin > best_d) {
        best_d = dmin;
        best_p = p;
        best_dir = d;
      }
      if (dmin >= 2.5) break;
    }
    bld.commit(k - 1, best_p, 1.5, 6, 4);
    prev_dir = best_dir;
  }
  std::vector<std::pair<int, int>> bonds;
  std::vector<double> r0;
  for (int k = 1; k < natom; k++) {
    bonds.push_back({k - 1, k});
    r0.push_back(1.5);
  }
  parameterise(rng, natom, bld.pos, bld.z, bonds, r0, noise, 110.0 * kPi / 180.0, false, out);
  return 0;
}

}  // namespace

extern "C" {

int sbsyn_make_molecule(uint64_t seed, int natom, double noise, int kind, sbsyn_molecule* out) {
  std::memset(out, 0, sizeof(sbsyn_molecule));
  if (natom < 2 || natom > 1000000) {
    return -1;
  }
  return (kind == 0) ? makeTree(seed, natom, noise, out) : makeChain(seed, natom, noise, out);
}

void sbsyn_free(sbsyn_molecule* m) {
  void* ptrs[] = {m->coords, m->charge, m->lj_idx, m->lja, m->ljb, m->z_numbers, m->mass,
                  m->pb_radii, m->gb_screen, m->bonds, m->bond_k, m->bond_r0, m->angles,
                  m->angl_k, m->angl_theta0, m->dihedrals, m->dihe_amp, m->dihe_freq,
                  m->dihe_phase, m->dihe_has14};
  for (void* p : ptrs) {
    std::free(p);
  }
  std::memset(m, 0, sizeof(sbsyn_molecule));
}

}  // extern "C"
