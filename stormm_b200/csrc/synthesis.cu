// Host side of the batched implicit-solvent path: builds the device layout of a synthesis of
// molecules (what STORMM's AtomGraphSynthesis, PhaseSpaceSynthesis, ImplicitSolventWorkspace and
// ScoreCard hold for this path), packs molecules into work units, and implements the C ABI of
// include/stormm_b200.h on top of the fused kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "stormm_b200.h"
#include "device_kits.h"
#include "synthesis.h"

namespace sb {

size_t fusedSmemBytes(int max_slots, int max_lj);
cudaError_t launchEvalFused(const DevSynthesis &d, int unit_begin, int unit_end, int max_lj,
                            int terms, bool force, bool energy, int blocks, int threads,
                            cudaStream_t stream, bool clash);
size_t minimizeSmemBytes(int max_slots, int max_lj);
cudaError_t launchMinimizerReset(const DevMinimizer &m, const DevSynthesis &d, double dx0,
                                 cudaStream_t stream);
cudaError_t launchMinimize(const DevSynthesis &d, const DevMinimizer &m, int unit_begin,
                           int unit_end, int max_lj, int cycles, bool final_energy, int threads,
                           int sm_count, cudaStream_t stream);
cudaError_t launchLineStep(const DevSynthesis &d, const DevMinimizer &m, int first, int count,
                           int step, cudaStream_t stream);
cudaError_t launchTiled(const DevSynthesis &d, const DevTiled &t, const int* h_tile_prefix,
                        const int* h_atom_prefix, int mol_begin, int mol_end, int terms,
                        bool force, bool energy, bool workspace, int sm_count,
                        cudaStream_t stream, bool clash);
cudaError_t launchTiled64(const DevSynthesis &d, const DevPrecise &p, const DevTiled &t,
                          const int* h_tile_prefix, const int* h_atom_prefix, int mol_begin,
                          int mol_end, int terms, bool force, bool energy, bool workspace,
                          int sm_count, cudaStream_t stream, bool clash);
cudaError_t launchImportCoordinates(const double* d_xyz, const int* d_map, int natom,
                                    double scale, long long* xcrd, long long* ycrd,
                                    long long* zcrd, int* xo, int* yo, int* zo, int* status,
                                    cudaStream_t stream);
cudaError_t launchExportCoordinates(const long long* xcrd, const long long* ycrd,
                                    const long long* zcrd, const int* d_map, int natom,
                                    double inv_scale, double* d_xyz, cudaStream_t stream);
cudaError_t launchExportForces(const long long* xf, const long long* yf, const long long* zf,
                               const int* xo, const int* yo, const int* zo, const int* d_map,
                               int natom, double inv_scale, double* d_xyz, cudaStream_t stream);
cudaError_t launchExportEnergies(const unsigned long long* nrg, int n, double inv_scale,
                                 double* d_out, cudaStream_t stream);
cudaError_t launchClear(const ClearList &list, int sm_count, cudaStream_t stream);
cudaError_t launchCharmmTerms(const DevCharmm &c, int ub0, int nub, int ci0, int nci, int cm0,
                              int ncm, bool force, bool energy, int sm_count,
                              cudaStream_t stream);
cudaError_t launchRestraints(const DevCharmm &c, int first, int count, bool force, bool energy,
                             int sm_count, cudaStream_t stream);
cudaError_t launchSurfaceArea(const long long* xcrd, const long long* ycrd,
                              const long long* zcrd, double inv_gpos_scale,
                              const int* atom_start, const int* atom_count, int nsys,
                              const double* radius, const double3* pts, int npts, double probe,
                              double weight, int* cell, double* out, cudaStream_t stream);

namespace {
thread_local std::string g_last_error;
}

cudaStream_t &allocationStream() {
  static thread_local cudaStream_t s = nullptr;
  return s;
}

void setLastError(const std::string &msg) { g_last_error = msg; }
const char* lastError() { return g_last_error.c_str(); }

void cudaCheck(cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    throw Error(SB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
  }
}

namespace {

double gbDefault(int igb, int which) {
  // Constants/generalized_born.h:52-75 (OBC-I, OBC-II, neck GB); HCT uses none of them, and neck
  // GB II takes its element-specific values from the topology
  if (igb == SB_GB_OBC) {
    return (which == 0) ? 0.8 : (which == 1) ? 0.0 : 2.909125;
  }
  if (igb == SB_GB_OBC2) {
    return (which == 0) ? 1.0 : (which == 1) ? 0.8 : 4.85;
  }
  if (igb == SB_GB_NECK) {
    return (which == 0) ? 1.09511284 : (which == 1) ? 1.90792938 : 2.50798245;
  }
  return 0.0;
}

uint32_t fbits(double v) {
  const float f = static_cast<float>(v);
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

}  // namespace

// Intrinsic radius -> row of the neck GB tables (Topology/atomgraph_setters.cpp:1088-1092)
static int neckIndex(double pb_radius) {
  return static_cast<int>(((pb_radius - 1.0) * 20.0) + 0.5);
}

void validateTopology(const sb_topology &tp, const sb_options &opt, int which) {
  const std::string name = (which >= 0) ? "topology " + std::to_string(which) : "the topology";
  if (tp.natom <= 0 || tp.natom > 65535 || tp.charge == nullptr || tp.lj_idx == nullptr ||
      tp.lja == nullptr || tp.ljb == nullptr || tp.n_lj_types <= 0 || tp.n_lj_types > 64) {
    throw Error(SB_ERR_ARGUMENT, name + " is incomplete or too large");
  }
  const int n = tp.natom;
  if (tp.nbond < 0 || tp.nangl < 0 || tp.ndihe < 0 ||
      (tp.nbond > 0 && (tp.bond_atoms == nullptr || tp.bond_keq == nullptr ||
                        tp.bond_leq == nullptr)) ||
      (tp.nangl > 0 && (tp.angl_atoms == nullptr || tp.angl_keq == nullptr ||
                        tp.angl_theta0 == nullptr)) ||
      (tp.ndihe > 0 && (tp.dihe_atoms == nullptr || tp.dihe_amp == nullptr ||
                        tp.dihe_freq == nullptr || tp.dihe_phase == nullptr))) {
    throw Error(SB_ERR_ARGUMENT, name + " has negative term counts or lacks term arrays");
  }
  for (int i = 0; i < n; i++) {
    if (tp.lj_idx[i] < 0 || tp.lj_idx[i] >= tp.n_lj_types) {
      throw Error(SB_ERR_ARGUMENT, name + ": Lennard-Jones type out of range");
    }
  }
  if (tp.excl_bounds != nullptr) {
    if (tp.excl_bounds[0] < 0 || (tp.excl_list == nullptr && tp.excl_bounds[n] > 0)) {
      throw Error(SB_ERR_ARGUMENT, name + ": exclusion bounds without an exclusion list");
    }
    for (int i = 0; i < n; i++) {
      if (tp.excl_bounds[i + 1] < tp.excl_bounds[i]) {
        throw Error(SB_ERR_ARGUMENT, name + ": exclusion bounds must not decrease");
      }
      for (int e = tp.excl_bounds[i]; e < tp.excl_bounds[i + 1]; e++) {
        if (tp.excl_list[e] < 0 || tp.excl_list[e] >= n) {
          throw Error(SB_ERR_ARGUMENT, name + ": exclusion partner out of range");
        }
      }
    }
  }
  if (opt.igb != SB_GB_NONE && (tp.pb_radii == nullptr || tp.gb_screen == nullptr)) {
    throw Error(SB_ERR_ARGUMENT, name + " lacks GB radii");
  }
  if (opt.igb == SB_GB_NECK || opt.igb == SB_GB_NECK2) {
    for (int i = 0; i < n; i++) {
      const int idx = neckIndex(tp.pb_radii[i]);
      if (idx < 0 || idx >= opt.neck_table_size) {
        throw Error(SB_ERR_ARGUMENT, name + ": neck GB needs intrinsic radii within the neck "
                    "tables (1-2 A for STORMM's 21 x 21 tables)");
      }
    }
    if (opt.igb == SB_GB_NECK2 && (tp.gb_alpha == nullptr || tp.gb_beta == nullptr ||
                                    tp.gb_gamma == nullptr)) {
      throw Error(SB_ERR_ARGUMENT, name + ": neck GB II takes element-specific alpha, beta and "
                  "gamma from the topology");
    }
  }
  auto in_range = [n](const int* atoms, size_t count) {
    for (size_t k = 0; k < count; k++) {
      if (atoms[k] < 0 || atoms[k] >= n) return false;
    }
    return true;
  };
  if (!in_range(tp.bond_atoms, 2 * static_cast<size_t>(tp.nbond)) ||
      !in_range(tp.angl_atoms, 3 * static_cast<size_t>(tp.nangl)) ||
      !in_range(tp.dihe_atoms, 4 * static_cast<size_t>(tp.ndihe))) {
    throw Error(SB_ERR_ARGUMENT, name + ": valence term atom index out of range");
  }
  // a dihedral's fourth atom shares its word with the improper flag
  for (int d = 0; d < tp.ndihe; d++) {
    if (tp.dihe_atoms[4 * d + 3] > 0x7fff) {
      throw Error(SB_ERR_UNSUPPORTED, name + ": dihedral atom index above 32767");
    }
  }
  // CHARMM terms
  if (tp.nubrd < 0 || tp.ncimp < 0 || tp.ncmap < 0 || tp.ncmap_surf < 0 ||
      (tp.nubrd > 0 && (tp.ubrd_atoms == nullptr || tp.ubrd_keq == nullptr ||
                        tp.ubrd_leq == nullptr)) ||
      (tp.ncimp > 0 && (tp.cimp_atoms == nullptr || tp.cimp_keq == nullptr ||
                        tp.cimp_phase == nullptr)) ||
      (tp.ncmap > 0 && (tp.cmap_atoms == nullptr || tp.cmap_surface == nullptr ||
                        tp.ncmap_surf <= 0 || tp.cmap_dims == nullptr ||
                        tp.cmap_values == nullptr))) {
    throw Error(SB_ERR_ARGUMENT, name + " has negative CHARMM term counts or lacks their arrays");
  }
  if (!in_range(tp.ubrd_atoms, 2 * static_cast<size_t>(tp.nubrd)) ||
      !in_range(tp.cimp_atoms, 4 * static_cast<size_t>(tp.ncimp)) ||
      !in_range(tp.cmap_atoms, 5 * static_cast<size_t>(tp.ncmap))) {
    throw Error(SB_ERR_ARGUMENT, name + ": CHARMM term atom index out of range");
  }
  if (tp.ncmap > 0) {
    for (int s = 0; s < tp.ncmap_surf; s++) {
      if (tp.cmap_dims[s] < 4 || tp.cmap_dims[s] > 360) {
        throw Error(SB_ERR_ARGUMENT, name + ": CMAP surface grids must have 4 to 360 points");
      }
    }
    for (int t = 0; t < tp.ncmap; t++) {
      if (tp.cmap_surface[t] < 0 || tp.cmap_surface[t] >= tp.ncmap_surf) {
        throw Error(SB_ERR_ARGUMENT, name + ": CMAP surface index out of range");
      }
    }
  }
}

namespace {

// First derivatives, per grid spacing, of the periodic cubic spline through n equally spaced
// values, as a stencil: the derivative at point i is sum_m w[m] y[(i + m) mod n].  The spline's
// knot slopes solve m[i-1] + 4 m[i] + m[i+1] = 3 (y[i+1] - y[i-1]) (continuous first and second
// derivatives, periodic), so w[m] = 3 (g[m-1] - g[m+1]) with g the first row of the inverse of
// that circulant matrix, found here by Gaussian elimination with partial pivoting.
std::vector<double> splineSlopeStencil(int n) {
  std::vector<double> a(static_cast<size_t>(n) * n, 0.0), g(n, 0.0);
  for (int i = 0; i < n; i++) {
    a[static_cast<size_t>(i) * n + i] = 4.0;
    a[static_cast<size_t>(i) * n + (i + 1) % n] += 1.0;
    a[static_cast<size_t>(i) * n + (i + n - 1) % n] += 1.0;
  }
  g[0] = 1.0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++) {
      if (std::fabs(a[static_cast<size_t>(r) * n + c]) > std::fabs(a[static_cast<size_t>(piv) * n + c])) piv = r;
    }
    if (piv != c) {
      for (int k = 0; k < n; k++) std::swap(a[static_cast<size_t>(c) * n + k], a[static_cast<size_t>(piv) * n + k]);
      std::swap(g[c], g[piv]);
    }
    for (int r = c + 1; r < n; r++) {
      const double f = a[static_cast<size_t>(r) * n + c] / a[static_cast<size_t>(c) * n + c];
      if (f == 0.0) continue;
      for (int k = c; k < n; k++) a[static_cast<size_t>(r) * n + k] -= f * a[static_cast<size_t>(c) * n + k];
      g[r] -= f * g[c];
    }
  }
  for (int r = n - 1; r >= 0; r--) {
    double v = g[r];
    for (int k = r + 1; k < n; k++) v -= a[static_cast<size_t>(r) * n + k] * g[k];
    g[r] = v / a[static_cast<size_t>(r) * n + r];
  }
  std::vector<double> w(n);
  for (int m = 0; m < n; m++) {
    w[m] = 3.0 * (g[(m + n - 1) % n] - g[(m + 1) % n]);
  }
  return w;
}

// The bicubic coefficients of every grid cell of one CMAP surface (value at phi index j, psi
// index k at j + k * n), appended to `out` cell by cell in the order j + k * n: for the cell at
// (j, k), with F the 4 x 4 matrix of values, phi slopes, psi slopes and cross slopes at its
// corners (rows: value and phi slope at j and j + 1; columns: value and psi slope at k and
// k + 1), the coefficients a[r + 4 s] of u^r v^s are M F M^T, M the cubic Hermite basis
// matrix; slopes per grid spacing from the periodic spline (Topology/atomgraph_refinement.cpp:
// 3307-3600 builds the same patches)
void cmapPatches(int n, const double* val, std::vector<double>* out) {
  const std::vector<double> w = splineSlopeStencil(n);
  auto at = [n](int j, int k) { return ((j % n) + n) % n + (((k % n) + n) % n) * n; };
  std::vector<double> dphi(static_cast<size_t>(n) * n), dpsi(dphi.size()), dcross(dphi.size());
  for (int k = 0; k < n; k++) {
    for (int j = 0; j < n; j++) {
      double sp = 0.0, ss = 0.0, sc = 0.0;
      for (int m = 0; m < n; m++) {
        sp += w[m] * val[at(j + m, k)];
        ss += w[m] * val[at(j, k + m)];
        for (int q = 0; q < n; q++) {
          sc += w[m] * w[q] * val[at(j + m, k + q)];
        }
      }
      dphi[at(j, k)] = sp;
      dpsi[at(j, k)] = ss;
      dcross[at(j, k)] = sc;
    }
  }
  static const double kM[4][4] = {{1.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 1.0, 0.0},
                                  {-3.0, 3.0, -2.0, -1.0}, {2.0, -2.0, 1.0, 1.0}};
  for (int k = 0; k < n; k++) {
    for (int j = 0; j < n; j++) {
      const int c00 = at(j, k), c10 = at(j + 1, k), c01 = at(j, k + 1), c11 = at(j + 1, k + 1);
      const double f[4][4] = {{val[c00], val[c01], dpsi[c00], dpsi[c01]},
                              {val[c10], val[c11], dpsi[c10], dpsi[c11]},
                              {dphi[c00], dphi[c01], dcross[c00], dcross[c01]},
                              {dphi[c10], dphi[c11], dcross[c10], dcross[c11]}};
      double mf[4][4];
      for (int r = 0; r < 4; r++) {
        for (int c = 0; c < 4; c++) {
          double v = 0.0;
          for (int q = 0; q < 4; q++) v += kM[r][q] * f[q][c];
          mf[r][c] = v;
        }
      }
      double cell[16];
      for (int r = 0; r < 4; r++) {
        for (int s = 0; s < 4; s++) {
          double v = 0.0;
          for (int q = 0; q < 4; q++) v += mf[r][q] * kM[s][q];
          cell[r + 4 * s] = v;
        }
      }
      out->insert(out->end(), cell, cell + 16);
    }
  }
}

}  // namespace

// CHARMM term records in the padded layout, system by system, and the CMAP surfaces of each
// topology once
void Synthesis::buildCharmm(const sb_topology* tops, int ntop) {
  h_ubrd.clear();
  h_ubrd_prm.clear();
  h_cimp.clear();
  h_cimp_sys.clear();
  h_cimp_prm.clear();
  h_cmap.clear();
  h_cmap_b.clear();
  h_cmap_surf.clear();
  h_cmap_patch.clear();
  h_ubrd_start.assign(nsys + 1, 0);
  h_cimp_start.assign(nsys + 1, 0);
  h_cmap_start.assign(nsys + 1, 0);
  std::vector<int> surf_base(ntop, -1);
  for (int s = 0; s < nsys; s++) {
    const int t = topo[s];
    const sb_topology &tp = tops[t];
    const int base = atom_start[s];
    for (int k = 0; k < tp.nubrd; k++) {
      h_ubrd.push_back(make_int4(base + tp.ubrd_atoms[2 * k], base + tp.ubrd_atoms[2 * k + 1], s, 0));
      h_ubrd_prm.push_back(make_double2(tp.ubrd_keq[k], tp.ubrd_leq[k]));
    }
    for (int k = 0; k < tp.ncimp; k++) {
      const int* a = tp.cimp_atoms + 4 * k;
      h_cimp.push_back(make_int4(base + a[0], base + a[1], base + a[2], base + a[3]));
      h_cimp_sys.push_back(s);
      h_cimp_prm.push_back(make_double2(tp.cimp_keq[k], tp.cimp_phase[k]));
    }
    if (tp.ncmap > 0 && surf_base[t] < 0) {
      surf_base[t] = static_cast<int>(h_cmap_surf.size());
      size_t vo = 0;
      for (int q = 0; q < tp.ncmap_surf; q++) {
        const int dim = tp.cmap_dims[q];
        h_cmap_surf.push_back(make_int2(static_cast<int>(h_cmap_patch.size() / 16), dim));
        cmapPatches(dim, tp.cmap_values + vo, &h_cmap_patch);
        vo += static_cast<size_t>(dim) * dim;
      }
    }
    for (int k = 0; k < tp.ncmap; k++) {
      const int* a = tp.cmap_atoms + 5 * k;
      h_cmap.push_back(make_int4(base + a[0], base + a[1], base + a[2], base + a[3]));
      h_cmap_b.push_back(make_int4(base + a[4], s, surf_base[t] + tp.cmap_surface[k], 0));
    }
    h_ubrd_start[s + 1] = static_cast<int>(h_ubrd.size());
    h_cimp_start[s + 1] = static_cast<int>(h_cimp.size());
    h_cmap_start[s + 1] = static_cast<int>(h_cmap.size());
  }
  has_charmm = !(h_ubrd.empty() && h_cimp.empty() && h_cmap.empty());
}

// The CHARMM terms and restraints of systems [first, last); cycle: the minimizer's per-system
// cycle counts, which then give the step of time-dependent restraints
void Synthesis::launchExtraTerms(int first, int last, bool force, bool energy,
                                 cudaStream_t stream, const int* cycle) {
  if (has_charmm) {
    cudaCheck(launchCharmmTerms(dev_charmm, h_ubrd_start[first],
                                h_ubrd_start[last] - h_ubrd_start[first], h_cimp_start[first],
                                h_cimp_start[last] - h_cimp_start[first], h_cmap_start[first],
                                h_cmap_start[last] - h_cmap_start[first], force, energy,
                                sm_count, stream),
              "CHARMM term launch");
  }
  if (!h_rst_start.empty() && h_rst_start[nsys] > 0) {
    DevCharmm c = dev_charmm;
    c.rst_cycle = cycle;
    cudaCheck(launchRestraints(c, h_rst_start[first],
                               h_rst_start[last] - h_rst_start[first], force, energy, sm_count,
                               stream),
              "restraint launch");
  }
}

// Restraints replace the previous set; records sorted by system so that a system's restraints
// are one contiguous range
void Synthesis::setRestraints(const sb_restraint* list, int count) {
  if (count < 0 || (count > 0 && list == nullptr)) {
    throw Error(SB_ERR_ARGUMENT, "restraints: negative count or no list");
  }
  std::vector<int> order(count);
  for (int q = 0; q < count; q++) {
    const sb_restraint &r = list[q];
    if (r.system < 0 || r.system >= nsys) {
      throw Error(SB_ERR_ARGUMENT, "restraint " + std::to_string(q) + ": system out of range");
    }
    if (r.kind < SB_RESTRAINT_POSITION || r.kind > SB_RESTRAINT_DIHEDRAL) {
      throw Error(SB_ERR_ARGUMENT, "restraint " + std::to_string(q) + ": unknown kind");
    }
    for (int m = 0; m < r.kind; m++) {
      if (r.atoms[m] < 0 || r.atoms[m] >= atom_count[r.system]) {
        throw Error(SB_ERR_ARGUMENT, "restraint " + std::to_string(q) + ": atom out of range");
      }
    }
    auto sane = [](double k2, double k3, double r1, double r2, double r3, double r4) {
      return r1 <= r2 && r2 <= r3 && r3 <= r4 && k2 >= 0.0 && k3 >= 0.0 && std::isfinite(r1) &&
             std::isfinite(r4) && std::isfinite(k2) && std::isfinite(k3);
    };
    const bool ramp = r.final_step != r.init_step;
    if (!sane(r.k2, r.k3, r.r1, r.r2, r.r3, r.r4) ||
        (ramp && !sane(r.final_k2, r.final_k3, r.final_r1, r.final_r2, r.final_r3,
                       r.final_r4))) {
      throw Error(SB_ERR_ARGUMENT, "restraint " + std::to_string(q) + ": bounds must ascend and "
                  "stiffnesses be finite and non-negative");
    }
    if (r.init_step < 0 || r.final_step < r.init_step) {
      throw Error(SB_ERR_ARGUMENT, "restraint " + std::to_string(q) + ": steps must satisfy "
                  "0 <= init_step <= final_step");
    }
    order[q] = q;
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return list[a].system < list[b].system; });
  std::vector<int4> atoms(count);
  std::vector<int2> meta(count);
  std::vector<double2> kk(count), kf(count);
  std::vector<double4> rr(count), tg(count), rf(count), tf(count);
  std::vector<int2> steps(count);
  h_rst_start.assign(nsys + 1, 0);
  for (int q = 0; q < count; q++) {
    const sb_restraint &r = list[order[q]];
    const int base = atom_start[r.system];
    int a[4];
    for (int m = 0; m < 4; m++) a[m] = base + ((m < r.kind) ? r.atoms[m] : r.atoms[0]);
    atoms[q] = make_int4(a[0], a[1], a[2], a[3]);
    meta[q] = make_int2(r.kind, r.system);
    kk[q] = make_double2(r.k2, r.k3);
    rr[q] = make_double4(r.r1, r.r2, r.r3, r.r4);
    tg[q] = make_double4(r.target[0], r.target[1], r.target[2], 0.0);
    steps[q] = make_int2(r.init_step, r.final_step);
    if (r.final_step != r.init_step) {
      kf[q] = make_double2(r.final_k2, r.final_k3);
      rf[q] = make_double4(r.final_r1, r.final_r2, r.final_r3, r.final_r4);
      tf[q] = make_double4(r.final_target[0], r.final_target[1], r.final_target[2], 0.0);
    }
    else {
      kf[q] = kk[q];
      rf[q] = rr[q];
      tf[q] = tg[q];
    }
    h_rst_start[r.system + 1]++;
  }
  for (int s = 0; s < nsys; s++) h_rst_start[s + 1] += h_rst_start[s];
  if (count > 0) {
    UploadArena arena;
    arena.put(&d_rst_atoms, atoms);
    arena.put(&d_rst_meta, meta);
    arena.put(&d_rst_k, kk);
    arena.put(&d_rst_r, rr);
    arena.put(&d_rst_target, tg);
    arena.put(&d_rst_kf, kf);
    arena.put(&d_rst_rf, rf);
    arena.put(&d_rst_target_f, tf);
    arena.put(&d_rst_steps, steps);
    arena.commit(&d_rst_arena);
  }
  dev_charmm.rst_atoms = d_rst_atoms.p;
  dev_charmm.rst_meta = d_rst_meta.p;
  dev_charmm.rst_k = d_rst_k.p;
  dev_charmm.rst_r = d_rst_r.p;
  dev_charmm.rst_target = d_rst_target.p;
  dev_charmm.rst_kf = d_rst_kf.p;
  dev_charmm.rst_rf = d_rst_rf.p;
  dev_charmm.rst_target_f = d_rst_target_f.p;
  dev_charmm.rst_steps = d_rst_steps.p;
  dev_charmm.xcrd = d_xcrd.p;
  dev_charmm.ycrd = d_ycrd.p;
  dev_charmm.zcrd = d_zcrd.p;
  dev_charmm.xfrc = d_xfrc.p;
  dev_charmm.yfrc = d_yfrc.p;
  dev_charmm.zfrc = d_zfrc.p;
  dev_charmm.energies = d_energies.p;
  dev_charmm.inv_gpos_scale = std::ldexp(1.0, -opt.gpos_bits);
  dev_charmm.frc_scale = std::ldexp(1.0, opt.frc_bits);
  dev_charmm.nrg_scale = std::ldexp(1.0, opt.nrg_bits);
  restraint_version++;
}

void UploadArena::commit(DeviceArray<unsigned char>* block) {
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  std::vector<size_t> up_at(up_.size()), zero_at(zero_.size());
  size_t up_bytes = 0;
  for (size_t k = 0; k < up_.size(); k++) {
    up_at[k] = up_bytes;
    up_bytes = align(up_bytes + up_[k].bytes);
  }
  size_t total = up_bytes;
  for (size_t k = 0; k < zero_.size(); k++) {
    zero_at[k] = total;
    total = align(total + zero_[k].bytes);
  }
  block->allocate(total > 0 ? total : 1);
  unsigned char* base = block->p;
  // the copy and the memset go on the block's allocation stream (the legacy default stream when
  // there is none) and are waited for here: the arrays are used next on other streams,
  // non-blocking ones among them, which do not order themselves after the default stream
  const cudaStream_t s = block->s;
  std::vector<unsigned char> host(up_bytes, 0);
  if (up_bytes > 0) {
    for (size_t k = 0; k < up_.size(); k++) {
      if (up_[k].src != nullptr) std::memcpy(host.data() + up_at[k], up_[k].src, up_[k].bytes);
    }
    cudaCheck(cudaMemcpyAsync(base, host.data(), up_bytes, cudaMemcpyHostToDevice, s),
              "cudaMemcpyAsync");
  }
  if (total > up_bytes) {
    cudaCheck(cudaMemsetAsync(base + up_bytes, 0, total - up_bytes, s), "cudaMemsetAsync");
  }
  cudaCheck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  for (size_t k = 0; k < up_.size(); k++) up_[k].bind(base + up_at[k]);
  for (size_t k = 0; k < zero_.size(); k++) zero_[k].bind(base + zero_at[k]);
  up_.clear();
  zero_.clear();
}

Synthesis::Synthesis(const sb_topology* tops, int ntop, const int* topology_index, int nsys_in,
                     const sb_options &options) :
    opt(options), nsys(nsys_in) {
  if (nsys <= 0 || ntop <= 0 || tops == nullptr || topology_index == nullptr) {
    throw Error(SB_ERR_ARGUMENT, "a synthesis needs at least one system and one topology");
  }
  if (opt.igb != SB_GB_NONE && opt.igb != SB_GB_HCT && opt.igb != SB_GB_OBC &&
      opt.igb != SB_GB_OBC2 && opt.igb != SB_GB_NECK && opt.igb != SB_GB_NECK2) {
    throw Error(SB_ERR_UNSUPPORTED, "implicit solvent model igb=" + std::to_string(opt.igb) +
                " is not available on this path (supported: 0, 1, 2, 5, 7, 8)");
  }
  // model constants of Potential/energy_abstracts.tpp:9-31
  neck = (opt.igb == SB_GB_NECK || opt.igb == SB_GB_NECK2);
  gb_offset = (opt.igb == SB_GB_NECK2) ? 0.195141 : 0.09;
  if (neck && (opt.neck_max_separation == nullptr || opt.neck_max_value == nullptr ||
               opt.neck_table_size < 1 || opt.neck_table_size > 64 || !(opt.neck_cut > 0.0))) {
    throw Error(SB_ERR_ARGUMENT, "neck GB needs the neck tables (size 1-64) and a positive cutoff");
  }
  if (opt.gpos_bits < 24 || opt.gpos_bits > 40 || opt.frc_bits < 18 || opt.frc_bits > 40 ||
      opt.nrg_bits < 22 || opt.nrg_bits > 40) {
    throw Error(SB_ERR_ARGUMENT, "fixed-point bit counts out of range");
  }
  if (opt.precision != SB_PRECISION_SINGLE && opt.precision != SB_PRECISION_DOUBLE) {
    throw Error(SB_ERR_ARGUMENT, "precision must be SB_PRECISION_SINGLE or SB_PRECISION_DOUBLE");
  }
  fp64 = (opt.precision == SB_PRECISION_DOUBLE);
  int dev_count = 0;
  cudaCheck(cudaGetDeviceCount(&dev_count), "cudaGetDeviceCount");
  if (opt.device < 0 || opt.device >= dev_count) {
    throw Error(SB_ERR_DEVICE, "CUDA device " + std::to_string(opt.device) + " not present");
  }
  cudaCheck(cudaSetDevice(opt.device), "cudaSetDevice");
  int major = 0;
  cudaCheck(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, opt.device),
            "cudaDeviceGetAttribute");
  if (major < 10) {
    throw Error(SB_ERR_DEVICE, "device " + std::to_string(opt.device) + " is not sm_100 class");
  }
  cudaCheck(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, opt.device),
            "cudaDeviceGetAttribute");
  cudaCheck(cudaDeviceGetAttribute(&max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                   opt.device), "cudaDeviceGetAttribute");

  topo.assign(topology_index, topology_index + nsys);
  for (int s = 0; s < nsys; s++) {
    if (topo[s] < 0 || topo[s] >= ntop) {
      throw Error(SB_ERR_ARGUMENT, "topology index out of range for system " + std::to_string(s));
    }
  }
  for (int t = 0; t < ntop; t++) {
    validateTopology(tops[t], opt, t);
  }
  buildLayout(tops, ntop);
  buildCharmm(tops, ntop);
  buildUnits();
  upload();
  // the caller's tables were copied; keep no pointer to them
  opt.neck_max_separation = nullptr;
  opt.neck_max_value = nullptr;
}

void Synthesis::buildLayout(const sb_topology* tops, int ntop) {
  const double sqrt_kc = std::sqrt(opt.coulomb_constant);
  atom_start.resize(nsys);
  atom_count.resize(nsys);
  int off = 0;
  for (int s = 0; s < nsys; s++) {
    atom_start[s] = off;
    atom_count[s] = tops[topo[s]].natom;
    off += (atom_count[s] + kTile - 1) / kTile * kTile;
  }
  natom_padded = off;
  natom_total = 0;
  h_unpadded_map.clear();
  for (int sy = 0; sy < nsys; sy++) {
    for (int i = 0; i < atom_count[sy]; i++) {
      h_unpadded_map.push_back(atom_start[sy] + i);
    }
    natom_total += atom_count[sy];
  }
  const size_t np = natom_padded;
  h_charge.assign(np, 0.0f);
  h_ljidx.assign(np, 0);
  h_sasa_radius.assign(np, 0.0);
  h_rho.assign(np, 1.0f);
  h_srho.assign(np, 0.0f);
  h_pb.assign(np, 1.09f);
  h_alpha.assign(np, 0.0f);
  h_beta.assign(np, 0.0f);
  h_gamma.assign(np, 0.0f);
  h_gb_radius64.assign(np, make_double4(1.0, 1.09, 0.0, 0.0));
  h_gb_gamma64.assign(np, 0.0);
  if (neck) {
    h_neck_idx.assign(np, 0);
    const size_t nt2 = static_cast<size_t>(opt.neck_table_size) * opt.neck_table_size;
    h64_neck_sep.assign(opt.neck_max_separation, opt.neck_max_separation + nt2);
    h64_neck_val.assign(opt.neck_max_value, opt.neck_max_value + nt2);
    h_neck_sep.assign(h64_neck_sep.begin(), h64_neck_sep.end());
    h_neck_val.assign(h64_neck_val.begin(), h64_neck_val.end());
  }
  if (fp64) {
    h64_charge.assign(np, 0.0);
    h64_rho.assign(np, 1.0);
    h64_srho.assign(np, 0.0);
    h64_pb.assign(np, 1.09);
    h64_alpha.assign(np, 0.0);
    h64_beta.assign(np, 0.0);
    h64_gamma.assign(np, 0.0);
  }

  // per-topology Lennard-Jones tables and tile exclusion masks
  std::vector<int> topo_lj_start(ntop), topo_tile_start(ntop);
  h_mask_pool.assign(32, 0u);   // mask 0: no exclusions
  for (int t = 0; t < ntop; t++) {
    const sb_topology &tp = tops[t];
    topo_lj_start[t] = h_ljab.size();
    const int nt = tp.n_lj_types;
    for (int e = 0; e < nt * nt; e++) {
      h_ljab.push_back(make_float2(static_cast<float>(tp.lja[e]), static_cast<float>(tp.ljb[e])));
      const double a14 = (tp.lja14 != nullptr) ? tp.lja14[e] : tp.lja[e];
      const double b14 = (tp.ljb14 != nullptr) ? tp.ljb14[e] : tp.ljb[e];
      h_ljab14.push_back(make_float2(static_cast<float>(a14), static_cast<float>(b14)));
      if (fp64) {
        h64_ljab14.push_back(make_double2(a14, b14));
        h64_ljab.push_back(make_double2(tp.lja[e], tp.ljb[e]));
      }
    }
    // exclusions as a symmetric set of pairs
    const int n = tp.natom;
    std::vector<std::vector<int>> partners(n);
    if (tp.excl_bounds != nullptr && tp.excl_list != nullptr) {
      for (int i = 0; i < n; i++) {
        for (int e = tp.excl_bounds[i]; e < tp.excl_bounds[i + 1]; e++) {
          const int j = tp.excl_list[e];
          if (j == i) continue;
          partners[i].push_back(j);
          partners[j].push_back(i);
        }
      }
    }
    const int nblk = (n + kTile - 1) / kTile;
    topo_tile_start[t] = h_tile_mask_idx.size();
    for (int I = 0; I < nblk; I++) {
      for (int J = 0; J <= I; J++) {
        // row l bit m: the pair (I*32 + l, J*32 + m) takes no Coulomb / Lennard-Jones term,
        // either because it is a 1-1..1-4 exclusion or because one of the slots is padding
        // beyond the molecule's last atom (as STORMM's tile masks mark them,
        // Potential/static_exclusionmask.cpp:120-150)
        unsigned rows[32] = {0u};
        bool any = false;
        for (int l = 0; l < kTile; l++) {
          const int a = I * kTile + l;
          if (a >= n) {
            rows[l] = 0xffffffffu;
            any = true;
            continue;
          }
          for (int m = 0; m < kTile; m++) {
            if (J * kTile + m >= n) {
              rows[l] |= (1u << m);
              any = true;
            }
          }
          for (int b : partners[a]) {
            if (b >= J * kTile && b < (J + 1) * kTile) {
              rows[l] |= (1u << (b - J * kTile));
              any = true;
            }
          }
        }
        if (any) {
          h_tile_mask_idx.push_back(static_cast<int>(h_mask_pool.size() / 32));
          h_mask_pool.insert(h_mask_pool.end(), rows, rows + 32);
        }
        else {
          h_tile_mask_idx.push_back(0);
        }
      }
    }
  }

  // per-system parameters and valence records
  h_lj_start.resize(nsys);
  h_lj_ntypes.resize(nsys);
  h_tile_start.resize(nsys);
  h_bond_start.assign(nsys + 1, 0);
  h_angl_start.assign(nsys + 1, 0);
  h_dihe_start.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; s++) {
    const int t = topo[s];
    const sb_topology &tp = tops[t];
    h_lj_start[s] = topo_lj_start[t];
    h_lj_ntypes[s] = tp.n_lj_types;
    h_tile_start[s] = topo_tile_start[t];
    const int base = atom_start[s];
    for (int i = 0; i < tp.natom; i++) {
      h_charge[base + i] = static_cast<float>(tp.charge[i] * sqrt_kc);
      h_ljidx[base + i] = tp.lj_idx[i];
      {
        // surface-area radius: half the sigma of the (type 0, atom type) entry of the pair
        // table, which is what STORMM's first n_lj_types sigma values hold
        const double a = tp.lja[tp.lj_idx[i]], b = tp.ljb[tp.lj_idx[i]];
        h_sasa_radius[base + i] = (b > 1.0e-6) ? 0.5 * std::sqrt(std::cbrt(a / b)) : 0.0;
      }
      if (opt.igb != SB_GB_NONE) {
        const double rho = tp.pb_radii[i] - gb_offset;
        h_rho[base + i] = static_cast<float>(rho);
        h_srho[base + i] = static_cast<float>(tp.gb_screen[i] * rho);
        h_pb[base + i] = static_cast<float>(tp.pb_radii[i]);
        h_alpha[base + i] = static_cast<float>(tp.gb_alpha ? tp.gb_alpha[i] : gbDefault(opt.igb, 0));
        h_beta[base + i] = static_cast<float>(tp.gb_beta ? tp.gb_beta[i] : gbDefault(opt.igb, 1));
        h_gamma[base + i] = static_cast<float>(tp.gb_gamma ? tp.gb_gamma[i] : gbDefault(opt.igb, 2));
        h_gb_radius64[base + i] = make_double4(
            rho, tp.pb_radii[i], tp.gb_alpha ? tp.gb_alpha[i] : gbDefault(opt.igb, 0),
            tp.gb_beta ? tp.gb_beta[i] : gbDefault(opt.igb, 1));
        h_gb_gamma64[base + i] = tp.gb_gamma ? tp.gb_gamma[i] : gbDefault(opt.igb, 2);
      }
      if (neck) {
        // AtomGraph::setImplicitSolventModel (Topology/atomgraph_setters.cpp:1088-1092)
        h_neck_idx[base + i] = neckIndex(tp.pb_radii[i]);
      }
      if (fp64) {
        h64_charge[base + i] = tp.charge[i] * sqrt_kc;
        if (opt.igb != SB_GB_NONE) {
          const double rho = tp.pb_radii[i] - gb_offset;
          h64_rho[base + i] = rho;
          h64_srho[base + i] = tp.gb_screen[i] * rho;
          h64_pb[base + i] = tp.pb_radii[i];
          h64_alpha[base + i] = tp.gb_alpha ? tp.gb_alpha[i] : gbDefault(opt.igb, 0);
          h64_beta[base + i] = tp.gb_beta ? tp.gb_beta[i] : gbDefault(opt.igb, 1);
          h64_gamma[base + i] = tp.gb_gamma ? tp.gb_gamma[i] : gbDefault(opt.igb, 2);
        }
      }
    }
    // indices were range-checked by validateTopology
    auto check_atom = [](int a) { return static_cast<uint32_t>(a); };
    for (int b = 0; b < tp.nbond; b++) {
      const uint32_t i = check_atom(tp.bond_atoms[2 * b]);
      const uint32_t j = check_atom(tp.bond_atoms[2 * b + 1]);
      const float leq_hi = static_cast<float>(tp.bond_leq[b]);
      h_bonds.push_back(make_uint4(i | (j << 16), fbits(tp.bond_keq[b]), fbits(leq_hi),
                                   fbits(tp.bond_leq[b] - static_cast<double>(leq_hi))));
      if (fp64) {
        h64_bond_atoms.push_back(make_int2(i, j));
        h64_bond_prm.push_back(make_double2(tp.bond_keq[b], tp.bond_leq[b]));
      }
    }
    h_bond_start[s + 1] = h_bonds.size();
    for (int a = 0; a < tp.nangl; a++) {
      const uint32_t i = check_atom(tp.angl_atoms[3 * a]);
      const uint32_t j = check_atom(tp.angl_atoms[3 * a + 1]);
      const uint32_t k = check_atom(tp.angl_atoms[3 * a + 2]);
      h_angles.push_back(make_uint4(i | (j << 16), k, fbits(tp.angl_keq[a]),
                                    fbits(std::cos(tp.angl_theta0[a]))));
      h_angl64.push_back(make_double4(tp.angl_keq[a], std::cos(tp.angl_theta0[a]),
                                      std::sin(tp.angl_theta0[a]), tp.angl_theta0[a]));
      if (fp64) {
        h64_angl_atoms.push_back(make_int4(i, j, k, 0));
        h64_angl_prm.push_back(make_double2(tp.angl_keq[a], tp.angl_theta0[a]));
      }
    }
    h_angl_start[s + 1] = h_angles.size();
    for (int d = 0; d < tp.ndihe; d++) {
      const uint32_t i = check_atom(tp.dihe_atoms[4 * d]);
      const uint32_t j = check_atom(tp.dihe_atoms[4 * d + 1]);
      const uint32_t k = check_atom(tp.dihe_atoms[4 * d + 2]);
      const uint32_t l = check_atom(tp.dihe_atoms[4 * d + 3]);
      const double scee = (tp.dihe_scee != nullptr) ? tp.dihe_scee[d] : 0.0;
      const double scnb = (tp.dihe_scnb != nullptr) ? tp.dihe_scnb[d] : 0.0;
      const uint32_t improper =
        (tp.dihe_improper != nullptr && tp.dihe_improper[d] != 0) ? 0x80000000u : 0u;
      h_dihe_a.push_back(make_uint4(i | (j << 16), k | (l << 16) | improper, fbits(tp.dihe_amp[d]),
                                    fbits(tp.dihe_freq[d])));
      h_dihe_b.push_back(make_uint4(fbits(std::cos(tp.dihe_phase[d])),
                                    fbits(std::sin(tp.dihe_phase[d])),
                                    fbits(scee > 0.0 ? 1.0 / scee : 0.0),
                                    fbits((scee > 0.0 && scnb > 0.0) ? 1.0 / scnb : 0.0)));
      h_dihe64.push_back(make_double4(tp.dihe_amp[d], std::cos(tp.dihe_phase[d]),
                                      std::sin(tp.dihe_phase[d]), tp.dihe_freq[d]));
      // the attached 1-4 pair's attenuated parameters in FP64, so that the kernel reads them
      // with the term instead of through a chain of dependent loads of charges, types and
      // tables: the same products the kernel formed from those (q_i q_l / scee, A / scnb,
      // B / scnb)
      if (scee > 0.0) {
        const double inv_scee = 1.0 / scee;
        const double inv_scnb = (scnb > 0.0) ? 1.0 / scnb : 0.0;
        const size_t e = static_cast<size_t>(tp.lj_idx[i]) * tp.n_lj_types + tp.lj_idx[l];
        const double a14 = (tp.lja14 != nullptr) ? tp.lja14[e] : tp.lja[e];
        const double b14 = (tp.ljb14 != nullptr) ? tp.ljb14[e] : tp.ljb[e];
        h_dihe14_64.push_back(make_double4((tp.charge[i] * sqrt_kc) * (tp.charge[l] * sqrt_kc) *
                                           inv_scee, a14 * inv_scnb, b14 * inv_scnb, 1.0));
      }
      else {
        h_dihe14_64.push_back(make_double4(0.0, 0.0, 0.0, 0.0));
      }
      if (fp64) {
        h64_dihe_atoms.push_back(make_int4(i, j, k, l));
        h64_dihe_prm.push_back(make_double4(tp.dihe_amp[d], tp.dihe_freq[d], tp.dihe_phase[d],
                                            improper ? 1.0 : 0.0));
        h64_dihe_attn.push_back(make_double2(scee > 0.0 ? 1.0 / scee : 0.0,
                                             (scee > 0.0 && scnb > 0.0) ? 1.0 / scnb : 0.0));
      }
    }
    h_dihe_start[s + 1] = h_dihe_a.size();
  }
}

std::unique_ptr<UnitPlan> Synthesis::makePlan(int max_slots_cap, int max_tiles_cap,
                                              bool defer) const {
  if (max_slots_cap < kTile || max_slots_cap % kTile != 0 || max_slots_cap > kMaxFusedAtoms ||
      max_tiles_cap < 1) {
    throw Error(SB_ERR_ARGUMENT, "work-unit caps must be a multiple of 32 atoms in [32, 2048] "
                "and at least one tile");
  }
  auto plan = std::make_unique<UnitPlan>();
  plan->max_slots_cap = max_slots_cap;
  plan->max_tiles_cap = max_tiles_cap;
  std::vector<int> order;
  for (int s = 0; s < nsys; s++) {
    if (atom_count[s] <= tiled_threshold) {
      order.push_back(s);   // molecules above the threshold take the tiled path
    }
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return atom_count[a] > atom_count[b]; });
  auto slots_of = [&](int s) { return (atom_count[s] + kTile - 1) / kTile * kTile; };
  auto tiles_of = [&](int s) {
    const int nb = (atom_count[s] + kTile - 1) / kTile;
    return nb * (nb + 1) / 2;
  };
  auto lj_of = [&](int s) { return 2 * h_lj_ntypes[s] * h_lj_ntypes[s]; };
  const int max_lj_cap = 2048;
  std::vector<int4> &units = plan->units;
  std::vector<int> &systems = plan->systems;
  // molecules above the packing cap: one unit each, at the front (largest first)
  size_t first_small = 0;
  while (first_small < order.size() && slots_of(order[first_small]) > max_slots_cap) {
    const int s = order[first_small];
    if (atom_count[s] > kMaxFusedAtoms) {
      throw Error(SB_ERR_UNSUPPORTED, "system " + std::to_string(s) + " has " +
                  std::to_string(atom_count[s]) + " atoms; the fused path holds up to " +
                  std::to_string(kMaxFusedAtoms) + " atoms per molecule");
    }
    units.push_back(make_int4(static_cast<int>(systems.size()), 1, slots_of(s), tiles_of(s)));
    systems.push_back(s);
    plan->big_slots = std::max(plan->big_slots, slots_of(s));
    plan->big_lj = std::max(plan->big_lj, lj_of(s));
    plan->n_big++;
    first_small++;
  }
  int4 cur = make_int4(static_cast<int>(systems.size()), 0, 0, 0);
  int cur_lj = 0;
  for (size_t oi = first_small; oi < order.size(); oi++) {
    const int s = order[oi];
    const bool fits = cur.y > 0 && cur.y < kMaxUnitSystems &&
                      cur.z + slots_of(s) <= max_slots_cap &&
                      cur.w + tiles_of(s) <= max_tiles_cap && cur_lj + lj_of(s) <= max_lj_cap;
    if (!fits && cur.y > 0) {
      units.push_back(cur);
      plan->small_lj = std::max(plan->small_lj, cur_lj);
      plan->small_slots = std::max(plan->small_slots, cur.z);
      cur = make_int4(static_cast<int>(systems.size()), 0, 0, 0);
      cur_lj = 0;
    }
    systems.push_back(s);
    cur.y++;
    cur.z += slots_of(s);
    cur.w += tiles_of(s);
    cur_lj += lj_of(s);
  }
  if (cur.y > 0) {
    units.push_back(cur);
    plan->small_lj = std::max(plan->small_lj, cur_lj);
    plan->small_slots = std::max(plan->small_slots, cur.z);
  }
  const size_t smem = fusedSmemBytes(std::max(plan->big_slots, plan->small_slots),
                                     std::max(plan->big_lj, plan->small_lj));
  if (static_cast<int>(smem) > max_smem_optin) {
    throw Error(SB_ERR_ARGUMENT, "work units need " + std::to_string(smem) +
                " bytes of shared memory, above the device limit");
  }
  finalizePlan(plan.get(), defer);
  return plan;
}

// Molecule table of every unit (what each block would otherwise rebuild serially) and the
// device descriptors pointing into it
void Synthesis::finalizePlan(UnitPlan* plan, bool defer) const {
  std::vector<int4> &desc = plan->desc;
  desc = plan->units;
  plan->meta.clear();
  int tile_base = 0;   // first tile of the unit in the pair-derivative store
  for (size_t u = 0; u < plan->units.size(); u++) {
    const int4 un = plan->units[u];
    desc[u].x = static_cast<int>(plan->meta.size() / kUnitMetaFields);
    int slot = 0, tile = 0, lj = 0, nb = 0, na = 0, nd = 0;
    bool fused = true;
    for (int k = 0; k < un.y; k++) {
      const int sid = plan->systems[un.x + k];
      fused = fused && (tiled_index[sid] < 0);
      const int n = atom_count[sid];
      const int nblk = (n + kTile - 1) / kTile;
      const int row[kUnitMetaFields] = {sid, n, slot, tile, lj, nb, na, nd};
      plan->meta.insert(plan->meta.end(), row, row + kUnitMetaFields);
      slot += nblk * kTile;
      tile += nblk * (nblk + 1) / 2;
      lj += 2 * h_lj_ntypes[sid] * h_lj_ntypes[sid];
      nb += (h_bond_start[sid + 1] - h_bond_start[sid] + 31) / 32;
      na += (h_angl_start[sid + 1] - h_angl_start[sid] + 31) / 32;
      nd += (h_dihe_start[sid + 1] - h_dihe_start[sid] + 31) / 32;
    }
    // closing row: the unit's first tile in the pair-derivative store, then the totals (units
    // of molecules on the tiled path never run the fused kernels and take no store)
    const int last[kUnitMetaFields] = {fused ? tile_base : 0, 0, slot, tile, lj, nb, na, nd};
    plan->meta.insert(plan->meta.end(), last, last + kUnitMetaFields);
    if (slot != un.z || tile != un.w) {
      throw Error(SB_ERR_ARGUMENT, "inconsistent work-unit descriptor");
    }
    if (fused) {
      tile_base += tile;
    }
  }
  if (tile_base > fused_tiles) {
    throw Error(SB_ERR_ARGUMENT, "work units hold more tiles than the molecules");
  }
  if (!defer) {
    plan->d_units.upload(desc);
    plan->d_meta.upload(plan->meta);
  }
}

void Synthesis::buildUnits() {
  threads = (opt.threads_per_block > 0) ? opt.threads_per_block : 256;
  if (threads % 32 != 0 || threads < 64 || threads > 256) {
    throw Error(SB_ERR_ARGUMENT, "threads per block must be a multiple of 32 in [64, 256]");
  }
  tiled_threshold = (opt.tiled_above_atoms > 0) ? opt.tiled_above_atoms : kMaxFusedAtoms;
  if (fp64) {
    tiled_threshold = 0;   // the FP64 mode evaluates every molecule tile by tile
  }
  else if (tiled_threshold < kTile || tiled_threshold > kMaxFusedAtoms) {
    throw Error(SB_ERR_ARGUMENT, "tiled_above_atoms must lie in [32, 2048]");
  }
  // molecules above the threshold: tiles of every one, in system order
  tiled_index.assign(nsys, -1);
  h_tiled_systems.clear();
  h_tile_prefix.assign(1, 0);
  h_atom_prefix.assign(1, 0);
  for (int s = 0; s < nsys; s++) {
    if (atom_count[s] > tiled_threshold) {
      const long long nb = (atom_count[s] + kTile - 1) / kTile;
      const long long tiles = static_cast<long long>(h_tile_prefix.back()) + nb * (nb + 1) / 2;
      if (tiles > 2000000000LL) {
        throw Error(SB_ERR_UNSUPPORTED, "too many tiles on the tiled path");
      }
      tiled_index[s] = static_cast<int>(h_tiled_systems.size());
      h_tiled_systems.push_back(s);
      h_tile_prefix.push_back(static_cast<int>(tiles));
      h_atom_prefix.push_back(h_atom_prefix.back() + static_cast<int>(nb) * kTile);
    }
  }
  long long ftiles = 0;
  for (int s = 0; s < nsys; s++) {
    if (tiled_index[s] < 0) {
      const long long nb = (atom_count[s] + kTile - 1) / kTile;
      ftiles += nb * (nb + 1) / 2;
    }
  }
  if (ftiles > 200000000LL) {
    throw Error(SB_ERR_UNSUPPORTED, "too many tiles on the fused path");
  }
  fused_tiles = static_cast<int>(ftiles);
  const int slots_cap = (opt.max_atoms_per_unit > 0) ? opt.max_atoms_per_unit : 256;
  // Default packing: molecules of four or fewer tiles share a unit, larger ones run alone
  // (measured on 1,024 molecules of 16-256 atoms: 213 us against 238 us for units packed up to
  // 36 tiles, which leave a sliver of a second wave)
  const int tiles_cap = (opt.max_tiles_per_unit > 0) ? opt.max_tiles_per_unit : 4;
  eval_plan = makePlan(slots_cap, tiles_cap, true);
  // minimization keeps whole molecules on chip for hundreds of cycles: smaller units balance
  // the persistent grid better (sb_autotune can choose another packing)
  min_plan = makePlan(128, 16, true);
  // one unit per system, in system order, for the per-system launches
  auto slots_of = [&](int s) { return (atom_count[s] + kTile - 1) / kTile * kTile; };
  auto tiles_of = [&](int s) {
    const int nb = (atom_count[s] + kTile - 1) / kTile;
    return nb * (nb + 1) / 2;
  };
  single_plan = std::make_unique<UnitPlan>();
  single_plan->units.resize(nsys);
  single_plan->systems.resize(nsys);
  single_slots = 0;
  single_lj = 0;
  for (int s = 0; s < nsys; s++) {
    single_plan->units[s] = make_int4(s, 1, slots_of(s), tiles_of(s));
    single_plan->systems[s] = s;
    if (tiled_index[s] < 0) {
      single_slots = std::max(single_slots, slots_of(s));
      single_lj = std::max(single_lj, 2 * h_lj_ntypes[s] * h_lj_ntypes[s]);
    }
  }
  max_unit_slots = single_slots;
  max_lj = single_lj;
  if (static_cast<int>(fusedSmemBytes(single_slots, single_lj)) > max_smem_optin) {
    throw Error(SB_ERR_ARGUMENT, "a molecule needs more shared memory than the device has");
  }
}

void Synthesis::upload() {
  // every array of the synthesis in one device block: one copy, one memset (UploadArena)
  UploadArena arena;
  finalizePlan(single_plan.get(), true);
  for (UnitPlan* plan : {eval_plan.get(), min_plan.get(), single_plan.get()}) {
    arena.put(&plan->d_units, plan->desc);
    arena.put(&plan->d_meta, plan->meta);
  }
  arena.put(&d_atom_start, atom_start);
  arena.put(&d_atom_count, atom_count);
  arena.put(&d_bond_start, h_bond_start);
  arena.put(&d_angl_start, h_angl_start);
  arena.put(&d_dihe_start, h_dihe_start);
  arena.put(&d_lj_start, h_lj_start);
  arena.put(&d_lj_ntypes, h_lj_ntypes);
  arena.put(&d_tile_start, h_tile_start);
  arena.put(&d_charge, h_charge);
  arena.put(&d_ljidx, h_ljidx);
  arena.put(&d_rho, h_rho);
  arena.put(&d_srho, h_srho);
  arena.put(&d_pb, h_pb);
  arena.put(&d_alpha, h_alpha);
  arena.put(&d_beta, h_beta);
  arena.put(&d_gamma, h_gamma);
  arena.put(&d_gb_radius64, h_gb_radius64);
  arena.put(&d_gb_gamma64, h_gb_gamma64);
  arena.put(&d_ljab, h_ljab);
  arena.put(&d_ljab14, h_ljab14);
  arena.put(&d_bonds, h_bonds);
  arena.put(&d_angles, h_angles);
  arena.put(&d_dihe_a, h_dihe_a);
  arena.put(&d_dihe_b, h_dihe_b);
  arena.put(&d_angl64, h_angl64);
  arena.put(&d_dihe64, h_dihe64);
  arena.put(&d_dihe14_64, h_dihe14_64);
  arena.put(&d_tile_mask_idx, h_tile_mask_idx);
  arena.put(&d_mask_pool, h_mask_pool);
  arena.put(&d_tiled_systems, h_tiled_systems);
  arena.put(&d_tile_prefix, h_tile_prefix);
  arena.put(&d_atom_prefix, h_atom_prefix);
  arena.put(&d_unpadded_map, h_unpadded_map);
  if (has_charmm) {
    arena.put(&d_ubrd, h_ubrd);
    arena.put(&d_ubrd_prm, h_ubrd_prm);
    arena.put(&d_cimp, h_cimp);
    arena.put(&d_cimp_sys, h_cimp_sys);
    arena.put(&d_cimp_prm, h_cimp_prm);
    arena.put(&d_cmap, h_cmap);
    arena.put(&d_cmap_b, h_cmap_b);
    arena.put(&d_cmap_surf, h_cmap_surf);
    arena.put(&d_cmap_patch, h_cmap_patch);
  }
  if (!h_tiled_systems.empty()) {
    arena.zero(&d_tiled_psi, natom_padded);
    arena.zero(&d_tiled_de, natom_padded);
    arena.zero(&d_tiled_radius, natom_padded);
    arena.zero(&d_tiled_sde, natom_padded);
  }
  if (fp64) {
    arena.put(&d64_charge, h64_charge);
    arena.put(&d64_ljab14, h64_ljab14);
    arena.put(&d64_rho, h64_rho);
    arena.put(&d64_srho, h64_srho);
    arena.put(&d64_pb, h64_pb);
    arena.put(&d64_alpha, h64_alpha);
    arena.put(&d64_beta, h64_beta);
    arena.put(&d64_gamma, h64_gamma);
    arena.put(&d64_ljab, h64_ljab);
    arena.put(&d64_bond_atoms, h64_bond_atoms);
    arena.put(&d64_bond_prm, h64_bond_prm);
    arena.put(&d64_angl_atoms, h64_angl_atoms);
    arena.put(&d64_angl_prm, h64_angl_prm);
    arena.put(&d64_dihe_atoms, h64_dihe_atoms);
    arena.put(&d64_dihe_prm, h64_dihe_prm);
    arena.put(&d64_dihe_attn, h64_dihe_attn);
    arena.zero(&d64_radius, natom_padded);
    arena.zero(&d64_sde, natom_padded);
    if (neck) {
      arena.put(&d64_neck_sep, h64_neck_sep);
      arena.put(&d64_neck_val, h64_neck_val);
    }
  }
  if (neck) {
    arena.put(&d_neck_idx, h_neck_idx);
    arena.put(&d_neck_sep, h_neck_sep);
    arena.put(&d_neck_val, h_neck_val);
  }
  const size_t np = natom_padded;
  arena.zero(&d_stage_xyz, static_cast<size_t>(3) * natom_total);
  arena.zero(&d_stage_nrg, static_cast<size_t>(nsys) * kNrgStride);
  arena.zero(&d_xcrd, np);
  arena.zero(&d_ycrd, np);
  arena.zero(&d_zcrd, np);
  arena.zero(&d_xcrd_ovrf, np);
  arena.zero(&d_ycrd_ovrf, np);
  arena.zero(&d_zcrd_ovrf, np);
  arena.zero(&d_xfrc, np);
  arena.zero(&d_yfrc, np);
  arena.zero(&d_zfrc, np);
  arena.zero(&d_xfrc_ovrf, np);
  arena.zero(&d_yfrc_ovrf, np);
  arena.zero(&d_zfrc_ovrf, np);
  arena.zero(&d_energies, static_cast<size_t>(nsys) * kNrgStride);
  arena.zero(&d_psi, np);
  arena.zero(&d_psi_ovrf, np);
  arena.zero(&d_sumdeijda, np);
  arena.zero(&d_sumdeijda_ovrf, np);
  arena.zero(&d_born_radii, np);
  arena.zero(&d_status, 1);
  // one tile beyond the last unit's, so no store or load of a tile walk can leave the buffer
  arena.zero(&d_pair_deriv, static_cast<size_t>(fused_tiles + 1) * kPairDerivPerTile);
  arena.commit(&d_arena);

  if (fp64) {
    dev64.charge = d64_charge.p;
    dev64.rho = d64_rho.p;
    dev64.srho = d64_srho.p;
    dev64.pb_radii = d64_pb.p;
    dev64.alpha = d64_alpha.p;
    dev64.beta = d64_beta.p;
    dev64.gamma = d64_gamma.p;
    dev64.ljab = d64_ljab.p;
    dev64.ljab14 = d64_ljab14.p;
    dev64.bond_atoms = d64_bond_atoms.p;
    dev64.bond_prm = d64_bond_prm.p;
    dev64.angl_atoms = d64_angl_atoms.p;
    dev64.angl_prm = d64_angl_prm.p;
    dev64.dihe_atoms = d64_dihe_atoms.p;
    dev64.dihe_prm = d64_dihe_prm.p;
    dev64.dihe_attn = d64_dihe_attn.p;
    dev64.kappa = (opt.saltcon > 1.0e-8) ? std::sqrt(0.10806 * opt.saltcon) : 0.0;
    dev64.inv_dielectric = 1.0 / opt.dielectric;
    dev64.radius = d64_radius.p;
    dev64.sde = d64_sde.p;
    dev64.gb_offset = gb_offset;
    if (neck) {
      dev64.neck_sep = d64_neck_sep.p;
      dev64.neck_val = d64_neck_val.p;
      dev64.neck_scale = (opt.igb == SB_GB_NECK2) ? 0.826836 : 0.361825;
      dev64.neck_cut = opt.neck_cut;
    }
  }
  dev_charmm = DevCharmm();
  if (has_charmm) {
    dev_charmm.ubrd = d_ubrd.p;
    dev_charmm.ubrd_prm = d_ubrd_prm.p;
    dev_charmm.cimp = d_cimp.p;
    dev_charmm.cimp_sys = d_cimp_sys.p;
    dev_charmm.cimp_prm = d_cimp_prm.p;
    dev_charmm.cmap = d_cmap.p;
    dev_charmm.cmap_b = d_cmap_b.p;
    dev_charmm.cmap_surf = d_cmap_surf.p;
    dev_charmm.cmap_patch = d_cmap_patch.p;
    dev_charmm.xcrd = d_xcrd.p;
    dev_charmm.ycrd = d_ycrd.p;
    dev_charmm.zcrd = d_zcrd.p;
    dev_charmm.xfrc = d_xfrc.p;
    dev_charmm.yfrc = d_yfrc.p;
    dev_charmm.zfrc = d_zfrc.p;
    dev_charmm.energies = d_energies.p;
    dev_charmm.inv_gpos_scale = std::ldexp(1.0, -opt.gpos_bits);
    dev_charmm.frc_scale = std::ldexp(1.0, opt.frc_bits);
    dev_charmm.nrg_scale = std::ldexp(1.0, opt.nrg_bits);
  }
  dev_tiled.nmol = static_cast<int>(h_tiled_systems.size());
  dev_tiled.ntiles = h_tile_prefix.back();
  dev_tiled.systems = d_tiled_systems.p;
  dev_tiled.tile_prefix = d_tile_prefix.p;
  dev_tiled.atom_prefix = d_atom_prefix.p;
  dev_tiled.psi_acc = d_tiled_psi.p;
  dev_tiled.de_acc = d_tiled_de.p;
  dev_tiled.radius = d_tiled_radius.p;
  dev_tiled.sde = d_tiled_sde.p;

  DevSynthesis &d = dev;
  std::memset(&d, 0, sizeof(DevSynthesis));
  d.nsys = nsys;
  d.natom_padded = natom_padded;
  d.igb = opt.igb;
  d.kappa = (opt.saltcon > 1.0e-8) ? static_cast<float>(std::sqrt(0.10806 * opt.saltcon)) : 0.0f;
  d.inv_dielectric = static_cast<float>(1.0 / opt.dielectric);
  d.frc_scale = static_cast<float>(std::ldexp(1.0, opt.frc_bits));
  d.nrg_scale = static_cast<float>(std::ldexp(1.0, opt.nrg_bits));
  d.inv_gpos_scale = std::ldexp(1.0, -opt.gpos_bits);
  d.psi_out_scale = std::ldexp(1.0, 24);
  d.atom_start = d_atom_start.p;
  d.atom_count = d_atom_count.p;
  d.bond_start = d_bond_start.p;
  d.angl_start = d_angl_start.p;
  d.dihe_start = d_dihe_start.p;
  d.lj_start = d_lj_start.p;
  d.lj_ntypes = d_lj_ntypes.p;
  d.tile_start = d_tile_start.p;
  d.xcrd = d_xcrd.p;
  d.ycrd = d_ycrd.p;
  d.zcrd = d_zcrd.p;
  d.xfrc = d_xfrc.p;
  d.yfrc = d_yfrc.p;
  d.zfrc = d_zfrc.p;
  d.xfrc_ovrf = d_xfrc_ovrf.p;
  d.yfrc_ovrf = d_yfrc_ovrf.p;
  d.zfrc_ovrf = d_zfrc_ovrf.p;
  d.charge = d_charge.p;
  d.lj_idx = d_ljidx.p;
  d.rho = d_rho.p;
  d.srho = d_srho.p;
  d.pb_radii = d_pb.p;
  d.gb_alpha = d_alpha.p;
  d.gb_beta = d_beta.p;
  d.gb_gamma = d_gamma.p;
  d.gb_radius64 = d_gb_radius64.p;
  d.gb_gamma64 = d_gb_gamma64.p;
  d.ljab = d_ljab.p;
  d.ljab14 = d_ljab14.p;
  d.bonds = d_bonds.p;
  d.angles = d_angles.p;
  d.dihe_a = d_dihe_a.p;
  d.dihe_b = d_dihe_b.p;
  d.angl64 = d_angl64.p;
  d.dihe64 = d_dihe64.p;
  d.dihe14_64 = d_dihe14_64.p;
  d.tile_mask_idx = d_tile_mask_idx.p;
  d.mask_pool = d_mask_pool.p;
  d.energies = d_energies.p;
  d.psi = d_psi.p;
  d.psi_ovrf = d_psi_ovrf.p;
  d.sumdeijda = d_sumdeijda.p;
  d.sumdeijda_ovrf = d_sumdeijda_ovrf.p;
  d.born_radii = d_born_radii.p;
  d.nunit = eval_plan->units.size();
  d.unit_desc = eval_plan->d_units.p;
  d.unit_meta = eval_plan->d_meta.p;
  d.max_unit_slots = max_unit_slots;
  d.pair_deriv = d_pair_deriv.p;
  d.gb_offset = static_cast<float>(gb_offset);
  if (neck) {
    d.neck_idx = d_neck_idx.p;
    d.neck_sep = d_neck_sep.p;
    d.neck_val = d_neck_val.p;
    d.neck_size = opt.neck_table_size;
    d.neck_scale = static_cast<float>((opt.igb == SB_GB_NECK2) ? 0.826836 : 0.361825);
    d.neck_cut = static_cast<float>(opt.neck_cut);
  }
  d.status = d_status.p;
}

void Synthesis::launchPlan(const UnitPlan &plan, int terms, bool force, bool energy,
                           cudaStream_t stream, const Clash &clash) {
  const int nunit = plan.units.size();
  DevSynthesis d = dev;
  d.nunit = nunit;
  d.unit_desc = plan.d_units.p;
  d.unit_meta = plan.d_meta.p;
  clash.apply(&d);
  if (plan.n_big > 0) {
    d.max_unit_slots = plan.big_slots;
    cudaCheck(launchEvalFused(d, 0, plan.n_big, plan.big_lj, terms, force, energy, plan.n_big,
                              launchThreads(plan.n_big, terms), stream, clash.on()),
              "fused evaluation launch (large molecules)");
  }
  if (nunit > plan.n_big) {
    d.max_unit_slots = plan.small_slots;
    cudaCheck(launchEvalFused(d, plan.n_big, nunit, plan.small_lj, terms, force, energy,
                              nunit - plan.n_big, launchThreads(nunit - plan.n_big, terms),
                              stream, clash.on()),
              "fused evaluation launch");
  }
}

// Threads a block for an evaluation launch of `units` work units: the configured count, or
// 512 when the launch evaluates every term and its units fit in one wave of 256-thread blocks
// (four an SM), where twice the warps on each unit finish the wave sooner (475 units of 16-256
// atoms: 141 us against 184); beyond one wave the 256-thread blocks are faster.  Sums are
// fixed-point, so the block size changes no result bit.
int Synthesis::launchThreads(int units, int terms) const {
  if (opt.threads_per_block > 0 || !allow_wide || terms != SB_TERM_ALL ||
      units >= 4 * sm_count) {
    return threads;
  }
  return 512;
}

void Synthesis::evaluate(int terms, bool force, bool energy, cudaStream_t stream,
                         const Clash &clash) {
  if (terms <= 0 || terms > SB_TERM_ALL) {
    throw Error(SB_ERR_ARGUMENT, "terms must be a nonzero mask of SB_TERM_*");
  }
  if (!force && !energy) {
    return;
  }
  launchPlan(*eval_plan, terms, force, energy, stream, clash);
  launchTiledRange(0, static_cast<int>(h_tiled_systems.size()), terms, force, energy, stream,
                   clash);
  if (terms & SB_TERM_VALENCE) {
    launchExtraTerms(0, nsys, force, energy, stream);
  }
}

void Synthesis::launchTiledRange(int mol_begin, int mol_end, int terms, bool force, bool energy,
                                 cudaStream_t stream, const Clash &clash) {
  if (mol_end <= mol_begin) {
    return;
  }
  const size_t np = natom_padded;
  cudaCheck(cudaMemsetAsync(d_tiled_psi.p, 0, np * sizeof(long long), stream), "memset");
  cudaCheck(cudaMemsetAsync(d_tiled_de.p, 0, np * sizeof(long long), stream), "memset");
  if (fp64) {
    DevPrecise p = dev64;
    p.clash_distance = clash.on() ? clash.distance64 : 0.0;
    p.clash_ratio = clash.on() ? clash.ratio64 : 0.0;
    p.clash_cycles = clash.cycles;
    p.clash_cycle = clash.cycle;
    cudaCheck(launchTiled64(dev, p, dev_tiled, h_tile_prefix.data(), h_atom_prefix.data(),
                            mol_begin, mol_end, terms, force, energy, true, sm_count, stream,
                            clash.on()),
              "FP64 evaluation launch");
    return;
  }
  DevSynthesis d = dev;
  clash.apply(&d);
  cudaCheck(launchTiled(d, dev_tiled, h_tile_prefix.data(), h_atom_prefix.data(), mol_begin,
                        mol_end, terms, force, energy, true, sm_count, stream, clash.on()),
            "tiled evaluation launch");
}

// The clash damping of the current minimization's evaluations: per system by its cycle count
Clash Synthesis::minimizerClash() const {
  Clash c;
  if (dev_min.clash_cycles > 0) {
    c.distance = dev_min.clash_distance;
    c.ratio = dev_min.clash_ratio;
    c.distance64 = min_clash_distance;
    c.ratio64 = min_clash_ratio;
    c.cycles = dev_min.clash_cycles;
    c.cycle = dev_min.cycle;
  }
  return c;
}

void Synthesis::rejectTiledMinimization(int kernel) const {
  if (fp64 && kernel != SB_MIN_GRAPH) {
    throw Error(SB_ERR_UNSUPPORTED, "the FP64 mode minimizes with the graph minimizer "
                "(SB_MIN_GRAPH) only");
  }
  if (!h_rst_start.empty() && h_rst_start[nsys] > 0 && kernel != SB_MIN_GRAPH) {
    throw Error(SB_ERR_UNSUPPORTED, "restraints are evaluated by a kernel of their own and "
                "cannot be minimized on chip by the persistent kernel; the graph minimizer "
                "(SB_MIN_GRAPH) minimizes them");
  }
  if (has_charmm && kernel != SB_MIN_GRAPH) {
    throw Error(SB_ERR_UNSUPPORTED, "CHARMM terms are evaluated by a kernel of their own and "
                "cannot be minimized on chip by the persistent kernel; the graph minimizer "
                "(SB_MIN_GRAPH) minimizes them");
  }
  if (!h_tiled_systems.empty() && kernel != SB_MIN_GRAPH) {
    throw Error(SB_ERR_UNSUPPORTED, "molecules above " + std::to_string(tiled_threshold) +
                " atoms are evaluated tile by tile and cannot be minimized on chip by the "
                "persistent kernel; the graph minimizer (SB_MIN_GRAPH) minimizes them");
  }
}

void Synthesis::evaluateRange(int first, int count, int terms, bool force, bool energy,
                              cudaStream_t stream, const Clash &clash) {
  if (first < 0 || count < 0 || first + count > nsys) {
    throw Error(SB_ERR_ARGUMENT, "system range out of bounds");
  }
  if (terms <= 0 || terms > SB_TERM_ALL) {
    throw Error(SB_ERR_ARGUMENT, "terms must be a nonzero mask of SB_TERM_*");
  }
  if (!force && !energy) {
    return;
  }
  DevSynthesis d = dev;
  d.unit_desc = single_plan->d_units.p;
  d.unit_meta = single_plan->d_meta.p;
  d.nunit = nsys;
  d.max_unit_slots = single_slots;
  clash.apply(&d);
  for (int s = first; s < first + count; s++) {
    if (tiled_index[s] >= 0) {
      launchTiledRange(tiled_index[s], tiled_index[s] + 1, terms, force, energy, stream, clash);
    }
    else {
      cudaCheck(launchEvalFused(d, s, s + 1, single_lj, terms, force, energy, 1, threads, stream,
                                clash.on()),
                "per-system evaluation launch");
    }
    if (terms & SB_TERM_VALENCE) {
      launchExtraTerms(s, s + 1, force, energy, stream);
    }
  }
}

void Synthesis::initialize(int what, cudaStream_t stream) {
  // every array to clear in one launch (all are multiples of 16 bytes: padded atom counts are
  // multiples of 32 and systems carry 16 energy slots); anything else falls back to a memset
  const size_t np = natom_padded;
  ClearList list;
  auto add = [&](void* p, size_t bytes) {
    if (bytes % 16 == 0 && list.count < 8) {
      list.ptr[list.count] = p;
      list.words[list.count] = bytes / 16;
      list.count++;
    }
    else {
      cudaCheck(cudaMemsetAsync(p, 0, bytes, stream), "memset");
    }
  };
  if (what & SB_INIT_FORCES) {
    add(d_xfrc.p, np * sizeof(long long));
    add(d_yfrc.p, np * sizeof(long long));
    add(d_zfrc.p, np * sizeof(long long));
    add(d_xfrc_ovrf.p, np * sizeof(int));
    add(d_yfrc_ovrf.p, np * sizeof(int));
    add(d_zfrc_ovrf.p, np * sizeof(int));
  }
  if (what & SB_INIT_ENERGIES) {
    add(d_energies.p, d_energies.n * sizeof(unsigned long long));
  }
  if (what & SB_INIT_GB_WORKSPACE) {
    ClearList first = list;
    if (list.count > 4) {
      cudaCheck(launchClear(first, sm_count, stream), "accumulator clear");
      list.count = 0;
    }
    add(d_psi.p, np * sizeof(long long));
    add(d_psi_ovrf.p, np * sizeof(int));
    add(d_sumdeijda.p, np * sizeof(long long));
    add(d_sumdeijda_ovrf.p, np * sizeof(int));
  }
  cudaCheck(launchClear(list, sm_count, stream), "accumulator clear");
}

void Synthesis::setCoordinates(const double* xyz, cudaStream_t stream) {
  // one copy of the caller's array (pinned memory makes it asynchronous and fast), then the
  // conversion to fixed point on the device; non-finite or out-of-range input sets bit 2 of
  // the status word and leaves those atoms unchanged
  cudaCheck(cudaMemcpyAsync(d_stage_xyz.p, xyz, sizeof(double) * 3 * natom_total,
                            cudaMemcpyHostToDevice, stream), "coordinate upload");
  cudaCheck(launchImportCoordinates(d_stage_xyz.p, d_unpadded_map.p, natom_total,
                                    std::ldexp(1.0, opt.gpos_bits), d_xcrd.p, d_ycrd.p,
                                    d_zcrd.p, d_xcrd_ovrf.p, d_ycrd_ovrf.p, d_zcrd_ovrf.p,
                                    d_status.p, stream), "coordinate import");
}

void Synthesis::getCoordinates(double* xyz, cudaStream_t stream) {
  cudaCheck(launchExportCoordinates(d_xcrd.p, d_ycrd.p, d_zcrd.p, d_unpadded_map.p, natom_total,
                                    std::ldexp(1.0, -opt.gpos_bits), d_stage_xyz.p, stream),
            "coordinate export");
  cudaCheck(cudaMemcpyAsync(xyz, d_stage_xyz.p, sizeof(double) * 3 * natom_total,
                            cudaMemcpyDeviceToHost, stream), "coordinate download");
  cudaCheck(cudaStreamSynchronize(stream), "coordinate download");
}

void Synthesis::getForcesFixed(long long* prim, int* ovrf, cudaStream_t stream) {
  const size_t np = natom_padded;
  cudaCheck(cudaMemcpyAsync(prim, d_xfrc.p, np * sizeof(long long), cudaMemcpyDeviceToHost,
                            stream), "force download");
  cudaCheck(cudaMemcpyAsync(prim + np, d_yfrc.p, np * sizeof(long long), cudaMemcpyDeviceToHost,
                            stream), "force download");
  cudaCheck(cudaMemcpyAsync(prim + 2 * np, d_zfrc.p, np * sizeof(long long),
                            cudaMemcpyDeviceToHost, stream), "force download");
  cudaCheck(cudaMemcpyAsync(ovrf, d_xfrc_ovrf.p, np * sizeof(int), cudaMemcpyDeviceToHost,
                            stream), "force download");
  cudaCheck(cudaMemcpyAsync(ovrf + np, d_yfrc_ovrf.p, np * sizeof(int), cudaMemcpyDeviceToHost,
                            stream), "force download");
  cudaCheck(cudaMemcpyAsync(ovrf + 2 * np, d_zfrc_ovrf.p, np * sizeof(int),
                            cudaMemcpyDeviceToHost, stream), "force download");
  cudaCheck(cudaStreamSynchronize(stream), "force download");
}

void Synthesis::getForces(double* xyz, cudaStream_t stream) {
  cudaCheck(launchExportForces(d_xfrc.p, d_yfrc.p, d_zfrc.p, d_xfrc_ovrf.p, d_yfrc_ovrf.p,
                               d_zfrc_ovrf.p, d_unpadded_map.p, natom_total,
                               std::ldexp(1.0, -opt.frc_bits), d_stage_xyz.p, stream),
            "force export");
  cudaCheck(cudaMemcpyAsync(xyz, d_stage_xyz.p, sizeof(double) * 3 * natom_total,
                            cudaMemcpyDeviceToHost, stream), "force download");
  cudaCheck(cudaStreamSynchronize(stream), "force download");
}

void Synthesis::getEnergiesFixed(long long* out, cudaStream_t stream) {
  cudaCheck(cudaMemcpyAsync(out, d_energies.p, d_energies.n * sizeof(long long),
                            cudaMemcpyDeviceToHost, stream), "energy download");
  cudaCheck(cudaStreamSynchronize(stream), "energy download");
}

void Synthesis::surfaceArea(const double* points, int npts, double probe, double weight,
                            double* out, cudaStream_t stream) {
  if (points == nullptr || out == nullptr || npts <= 0 || !(probe >= 0.0) ||
      !std::isfinite(probe) || !std::isfinite(weight)) {
    throw Error(SB_ERR_ARGUMENT, "surface area: points, a positive point count, a finite "
                "non-negative probe and a finite weight are required");
  }
  std::vector<double3> pts(npts);
  for (int p = 0; p < npts; p++) {
    pts[p] = make_double3(points[3 * p], points[3 * p + 1], points[3 * p + 2]);
  }
  DeviceArray<double> radius, result;
  DeviceArray<double3> d_pts;
  DeviceArray<int> cell;
  radius.allocate(h_sasa_radius.size());
  d_pts.allocate(npts);
  cell.allocate(h_sasa_radius.size());
  result.allocate(nsys);
  cudaCheck(cudaMemcpyAsync(radius.p, h_sasa_radius.data(), h_sasa_radius.size() * sizeof(double),
                            cudaMemcpyHostToDevice, stream), "surface area upload");
  cudaCheck(cudaMemcpyAsync(d_pts.p, pts.data(), npts * sizeof(double3), cudaMemcpyHostToDevice,
                            stream), "surface area upload");
  cudaCheck(launchSurfaceArea(d_xcrd.p, d_ycrd.p, d_zcrd.p, std::ldexp(1.0, -opt.gpos_bits),
                              d_atom_start.p, d_atom_count.p, nsys, radius.p, d_pts.p, npts,
                              probe, weight, cell.p, result.p, stream), "surface area launch");
  cudaCheck(cudaMemcpyAsync(out, result.p, nsys * sizeof(double), cudaMemcpyDeviceToHost,
                            stream), "surface area download");
  cudaCheck(cudaStreamSynchronize(stream), "surface area");
}

void Synthesis::getEnergies(double* out, cudaStream_t stream) {
  const int n = nsys * kNrgStride;
  cudaCheck(launchExportEnergies(d_energies.p, n, std::ldexp(1.0, -opt.nrg_bits), d_stage_nrg.p,
                                 stream), "energy export");
  cudaCheck(cudaMemcpyAsync(out, d_stage_nrg.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                            stream), "energy download");
  cudaCheck(cudaStreamSynchronize(stream), "energy download");
}

// Forces and energies exported and copied into the caller's page-locked buffers on the stream,
// without waiting: a serving loop overlaps one batch's copies with another's evaluation
void Synthesis::downloadResults(double* forces, double* energies, cudaStream_t stream) {
  for (const double* p : {static_cast<const double*>(forces), static_cast<const double*>(energies)}) {
    if (p == nullptr) continue;
    cudaPointerAttributes attr;
    cudaCheck(cudaPointerGetAttributes(&attr, p), "cudaPointerGetAttributes");
    if (attr.type != cudaMemoryTypeHost) {
      throw Error(SB_ERR_ARGUMENT, "asynchronous downloads need page-locked host buffers");
    }
  }
  if (forces != nullptr) {
    cudaCheck(launchExportForces(d_xfrc.p, d_yfrc.p, d_zfrc.p, d_xfrc_ovrf.p, d_yfrc_ovrf.p,
                                 d_zfrc_ovrf.p, d_unpadded_map.p, natom_total,
                                 std::ldexp(1.0, -opt.frc_bits), d_stage_xyz.p, stream),
              "force export");
    cudaCheck(cudaMemcpyAsync(forces, d_stage_xyz.p, sizeof(double) * 3 * natom_total,
                              cudaMemcpyDeviceToHost, stream), "force download");
  }
  if (energies != nullptr) {
    const int n = nsys * kNrgStride;
    cudaCheck(launchExportEnergies(d_energies.p, n, std::ldexp(1.0, -opt.nrg_bits),
                                   d_stage_nrg.p, stream), "energy export");
    cudaCheck(cudaMemcpyAsync(energies, d_stage_nrg.p, sizeof(double) * n,
                              cudaMemcpyDeviceToHost, stream), "energy download");
  }
}

void Synthesis::getGbWorkspace(double* psi, double* radii, double* sde, cudaStream_t stream) {
  const size_t np = natom_padded;
  std::vector<long long> p(np), q(np);
  std::vector<float> r(np);
  cudaCheck(cudaMemcpyAsync(p.data(), d_psi.p, np * sizeof(long long), cudaMemcpyDeviceToHost,
                            stream), "workspace download");
  cudaCheck(cudaMemcpyAsync(q.data(), d_sumdeijda.p, np * sizeof(long long),
                            cudaMemcpyDeviceToHost, stream), "workspace download");
  cudaCheck(cudaMemcpyAsync(r.data(), d_born_radii.p, np * sizeof(float), cudaMemcpyDeviceToHost,
                            stream), "workspace download");
  cudaCheck(cudaStreamSynchronize(stream), "workspace download");
  const double inv = std::ldexp(1.0, -24);
  size_t dst = 0;
  for (int s = 0; s < nsys; s++) {
    for (int i = 0; i < atom_count[s]; i++) {
      const size_t a = atom_start[s] + i;
      if (psi) psi[dst] = static_cast<double>(p[a]) * inv;
      if (sde) sde[dst] = static_cast<double>(q[a]) * inv;
      if (radii) radii[dst] = r[a];
      dst++;
    }
  }
}

int Synthesis::checkStatus(cudaStream_t stream) {
  int st = 0;
  cudaCheck(cudaMemcpyAsync(&st, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, stream),
            "status download");
  cudaCheck(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream), "status reset");
  cudaCheck(cudaStreamSynchronize(stream), "status download");
  return st;
}

// ------------------------------------------------------------------------------------------------
// Line minimization (MolecularMechanics/hpc_minimization.cu:129-600)
// ------------------------------------------------------------------------------------------------
void validateMinimizeControls(const sb_minimize_controls &ctl) {
  if (ctl.total_cycles < 0 || ctl.sd_cycles < 0) {
    throw Error(SB_ERR_ARGUMENT, "cycle counts must not be negative");
  }
  if (ctl.clash_cycles < 0 || !(ctl.clash_distance >= 0.0) || !(ctl.clash_ratio >= 0.0) ||
      !std::isfinite(ctl.clash_distance) || !std::isfinite(ctl.clash_ratio)) {
    throw Error(SB_ERR_ARGUMENT, "clash-damping cycles, distance and ratio must not be negative");
  }
  if (!(ctl.initial_step > 0.0) || !std::isfinite(ctl.initial_step) ||
      !(ctl.convergence_rms >= 0.0)) {
    throw Error(SB_ERR_ARGUMENT, "initial step must be positive and the RMS target not negative");
  }
  if (ctl.kernel != SB_MIN_GRAPH && ctl.kernel != SB_MIN_PERSISTENT) {
    throw Error(SB_ERR_ARGUMENT, "unknown minimization kernel choice");
  }
}

void Synthesis::minimizeBegin(const sb_minimize_controls &ctl, cudaStream_t stream) {
  validateMinimizeControls(ctl);
  rejectTiledMinimization(ctl.kernel);
  const size_t np = natom_padded;
  if (d_mcycle.p == nullptr) {
    // the minimizer's arrays in one block (every kernel that reads them writes them first)
    UploadArena arena;
    arena.zero(&d_xprv, np);
    arena.zero(&d_yprv, np);
    arena.zero(&d_zprv, np);
    arena.zero(&d_xcg, np);
    arena.zero(&d_ycg, np);
    arena.zero(&d_zcg, np);
    arena.zero(&d_lmove, nsys);
    arena.zero(&d_rmsf, nsys);
    arena.zero(&d_mcycle, nsys);
    arena.zero(&d_mdone, nsys);
    arena.zero(&d_line, static_cast<size_t>(nsys) * kLineFields);
    arena.zero(&d_queue, 2);
    if (fp64) {
      arena.zero(&d_xcg64, np);
      arena.zero(&d_ycg64, np);
      arena.zero(&d_zcg64, np);
    }
    arena.commit(&d_min_arena);
  }
  history_stride = 0;
  if (ctl.record_history) {
    history_stride = ctl.total_cycles + 1;
    const size_t need = static_cast<size_t>(nsys) * history_stride;
    if (d_history.n < need) {
      d_history.allocate(need);
    }
    cudaCheck(cudaMemsetAsync(d_history.p, 0, need * sizeof(double), stream), "memset");
  }
  DevMinimizer &m = dev_min;
  std::memset(&m, 0, sizeof(DevMinimizer));
  m.xcrd = d_xcrd.p;
  m.ycrd = d_ycrd.p;
  m.zcrd = d_zcrd.p;
  m.xprv = d_xprv.p;
  m.yprv = d_yprv.p;
  m.zprv = d_zprv.p;
  m.xcg = d_xcg.p;
  m.ycg = d_ycg.p;
  m.zcg = d_zcg.p;
  if (fp64) {
    m.xcg64 = d_xcg64.p;
    m.ycg64 = d_ycg64.p;
    m.zcg64 = d_zcg64.p;
  }
  m.l_move = d_lmove.p;
  m.cycle = d_mcycle.p;
  m.done = d_mdone.p;
  m.rms_force = d_rmsf.p;
  m.history = ctl.record_history ? d_history.p : nullptr;
  m.hist_stride = history_stride;
  m.sd_cycles = ctl.sd_cycles;
  m.max_cycles = ctl.total_cycles;
  m.drms = ctl.convergence_rms;
  min_clash_distance = 0.0;
  min_clash_ratio = 0.0;
  if (ctl.clash_cycles > 0 && (ctl.clash_distance > 0.0 || ctl.clash_ratio > 0.0)) {
    m.clash_cycles = ctl.clash_cycles;
    m.clash_distance = static_cast<float>(ctl.clash_distance);
    min_clash_distance = ctl.clash_distance;
    min_clash_ratio = ctl.clash_ratio;
    m.clash_ratio = static_cast<float>(ctl.clash_ratio);
  }
  m.queue = d_queue.p;
  m.line = d_line.p;
  min_kernel = ctl.kernel;
  min_total_cycles = ctl.total_cycles;
  cudaCheck(launchMinimizerReset(m, dev, ctl.initial_step, stream), "minimizer reset");
  min_ready = true;
}

Synthesis::~Synthesis() {
  if (cycle_graph != nullptr) {
    cudaGraphExecDestroy(cycle_graph);
  }
  if (capture_stream != nullptr) {
    cudaStreamDestroy(capture_stream);
  }
}

// One batched evaluation of all systems (single = false) or of systems [first, first + count)
// one launch each (single = true); molecules above the on-chip limit go tile by tile
void Synthesis::evaluateFor(int first, int count, bool single, bool force, cudaStream_t stream,
                            const Clash &clash) {
  if (!single) {
    launchPlan(*eval_plan, SB_TERM_ALL, force, true, stream, clash);
    launchTiledRange(0, static_cast<int>(h_tiled_systems.size()), SB_TERM_ALL, force, true,
                     stream, clash);
    launchExtraTerms(0, nsys, force, true, stream, dev_min.cycle);
    return;
  }
  DevSynthesis d = dev;
  d.unit_desc = single_plan->d_units.p;
  d.unit_meta = single_plan->d_meta.p;
  d.nunit = nsys;
  d.max_unit_slots = single_slots;
  clash.apply(&d);
  for (int s = first; s < first + count; s++) {
    if (tiled_index[s] >= 0) {
      launchTiledRange(tiled_index[s], tiled_index[s] + 1, SB_TERM_ALL, force, true, stream,
                       clash);
    }
    else {
      cudaCheck(launchEvalFused(d, s, s + 1, single_lj, SB_TERM_ALL, force, true, 1, threads,
                                stream, clash.on()), "per-system evaluation launch");
    }
    launchExtraTerms(s, s + 1, force, true, stream, dev_min.cycle);
  }
}

// One graph-mode cycle: evaluations by the batched evaluation kernel, line-search steps by a warp
// per system (line_search.cu)
void Synthesis::graphCycle(int first, int count, bool single, cudaStream_t stream) {
  const size_t nrg_bytes = d_energies.n * sizeof(unsigned long long);
  const Clash clash = minimizerClash();
  initialize(SB_INIT_FORCES | SB_INIT_ENERGIES, stream);
  evaluateFor(first, count, single, true, stream, clash);
  cudaCheck(launchLineStep(dev, dev_min, first, count, 0, stream), "line search launch");
  for (int step = 1; step <= 3; step++) {
    cudaCheck(cudaMemsetAsync(d_energies.p, 0, nrg_bytes, stream), "memset");
    evaluateFor(first, count, single, false, stream, clash);
    cudaCheck(launchLineStep(dev, dev_min, first, count, step, stream), "line search launch");
  }
}

// Energies at the coordinates reached, and their history entry
void Synthesis::graphFinalEnergy(int first, int count, bool single, cudaStream_t stream) {
  cudaCheck(cudaMemsetAsync(d_energies.p, 0, d_energies.n * sizeof(unsigned long long), stream),
            "memset");
  evaluateFor(first, count, single, false, stream);
  cudaCheck(launchLineStep(dev, dev_min, first, count, 4, stream), "line search launch");
}

void Synthesis::launchMinPlan(const UnitPlan &plan, int cycles, bool final_energy,
                              cudaStream_t stream) {
  DevMinimizer m = dev_min;
  cudaCheck(cudaMemsetAsync(d_queue.p, 0, 2 * sizeof(int), stream), "memset");
  const int nunit = plan.units.size();
  DevSynthesis d = dev;
  d.nunit = nunit;
  d.unit_desc = plan.d_units.p;
  d.unit_meta = plan.d_meta.p;
  if (plan.n_big > 0) {
    d.max_unit_slots = plan.big_slots;
    m.queue = d_queue.p;
    if (static_cast<int>(minimizeSmemBytes(plan.big_slots, plan.big_lj)) > max_smem_optin) {
      throw Error(SB_ERR_UNSUPPORTED, "a molecule is too large for on-chip minimization");
    }
    cudaCheck(launchMinimize(d, m, 0, plan.n_big, plan.big_lj, cycles, final_energy, threads,
                             sm_count, stream), "minimization launch (large molecules)");
  }
  if (nunit > plan.n_big) {
    d.max_unit_slots = plan.small_slots;
    m.queue = d_queue.p + 1;
    cudaCheck(launchMinimize(d, m, plan.n_big, nunit, plan.small_lj, cycles, final_energy,
                             threads, sm_count, stream), "minimization launch");
  }
}

// The line-search steps one at a time, for a caller that runs its own evaluations between them
// (STORMM's launchConjugateGradient and launchLineAdvance): every system of the synthesis
void Synthesis::conjugateGradient(cudaStream_t stream) {
  if (!min_ready) {
    throw Error(SB_ERR_ARGUMENT, "no minimization has begun on this synthesis");
  }
  cudaCheck(launchLineStep(dev, dev_min, 0, nsys, 5, stream), "conjugate gradient launch");
}

void Synthesis::lineAdvance(int move, cudaStream_t stream) {
  if (!min_ready) {
    throw Error(SB_ERR_ARGUMENT, "no minimization has begun on this synthesis");
  }
  if (move < 0 || move > 3) {
    throw Error(SB_ERR_ARGUMENT, "line move number must be 0, 1, 2 or 3");
  }
  cudaCheck(launchLineStep(dev, dev_min, 0, nsys, (move == 0) ? 6 : move, stream),
            "line advance launch");
}

void Synthesis::minimizeAdvance(int cycles, bool final_energy, cudaStream_t stream) {
  if (!min_ready) {
    throw Error(SB_ERR_ARGUMENT, "no minimization has begun on this synthesis");
  }
  if (cycles < 0) {
    throw Error(SB_ERR_ARGUMENT, "cycle count must not be negative");
  }
  if (min_kernel == SB_MIN_PERSISTENT) {
    launchMinPlan(*min_plan, cycles, final_energy, stream);
    return;
  }
  if (cycles > 0) {
    // the graph holds its kernels' arguments by value: capture again when any of them changed
    const bool stale = cycle_graph == nullptr || cycle_graph_plan != eval_plan.get() ||
                       std::memcmp(&cycle_graph_min, &dev_min, sizeof(DevMinimizer)) != 0 ||
                       std::memcmp(&cycle_graph_dev, &dev, sizeof(DevSynthesis)) != 0 ||
                       cycle_graph_restraints != restraint_version;
    if (stale) {
      // capture one cycle on a stream of the synthesis' own, then replay it on the caller's
      if (cycle_graph != nullptr) {
        cudaCheck(cudaGraphExecDestroy(cycle_graph), "cudaGraphExecDestroy");
        cycle_graph = nullptr;
      }
      if (capture_stream == nullptr) {
        cudaCheck(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking),
                  "cudaStreamCreate");
      }
      cudaCheck(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeRelaxed),
                "cudaStreamBeginCapture");
      cudaGraph_t graph = nullptr;
      try {
        graphCycle(0, nsys, false, capture_stream);
      }
      catch (...) {
        cudaStreamEndCapture(capture_stream, &graph);
        if (graph != nullptr) cudaGraphDestroy(graph);
        throw;
      }
      cudaCheck(cudaStreamEndCapture(capture_stream, &graph), "cudaStreamEndCapture");
      const cudaError_t err = cudaGraphInstantiate(&cycle_graph, graph, 0);
      cudaGraphDestroy(graph);
      cudaCheck(err, "cudaGraphInstantiate");
      cycle_graph_plan = eval_plan.get();
      cycle_graph_min = dev_min;
      cycle_graph_dev = dev;
      cycle_graph_restraints = restraint_version;
    }
    for (int c = 0; c < cycles; c++) {
      cudaCheck(cudaGraphLaunch(cycle_graph, stream), "cudaGraphLaunch");
    }
  }
  if (final_energy) {
    graphFinalEnergy(0, nsys, false, stream);
  }
}

void Synthesis::minimize(const sb_minimize_controls &ctl, cudaStream_t stream) {
  minimizeBegin(ctl, stream);
  minimizeAdvance(ctl.total_cycles, true, stream);
}

void Synthesis::minimizeRange(int first, int count, const sb_minimize_controls &ctl,
                              cudaStream_t stream) {
  if (first < 0 || count < 0 || first + count > nsys) {
    throw Error(SB_ERR_ARGUMENT, "system range out of bounds");
  }
  minimizeBegin(ctl, stream);
  if (min_kernel == SB_MIN_GRAPH) {
    // the per-system sequence: every launch of every cycle for one system at a time
    for (int s = first; s < first + count; s++) {
      for (int c = 0; c < ctl.total_cycles; c++) {
        graphCycle(s, 1, true, stream);
      }
    }
    graphFinalEnergy(first, count, true, stream);
    return;
  }
  DevSynthesis d = dev;
  d.unit_desc = single_plan->d_units.p;
  d.unit_meta = single_plan->d_meta.p;
  d.nunit = nsys;
  d.max_unit_slots = single_slots;
  if (static_cast<int>(minimizeSmemBytes(single_slots, single_lj)) > max_smem_optin) {
    throw Error(SB_ERR_UNSUPPORTED, "a molecule is too large for on-chip minimization");
  }
  // one block per launch: the unit counter is never consulted for a second unit
  for (int s = first; s < first + count; s++) {
    cudaCheck(launchMinimize(d, dev_min, s, s + 1, single_lj, ctl.total_cycles, true, threads,
                             sm_count, stream), "per-system minimization launch");
  }
}

// ------------------------------------------------------------------------------------------------
// Autotuning of the work-unit packing (in place of CoreKlManager's fixed launch tables,
// Structure/core_kernel_manager.cpp:538-600).  Results do not depend on the packing (every sum
// is per molecule and order-independent), so the fastest candidate is simply kept.
// ------------------------------------------------------------------------------------------------
void Synthesis::autotune(int what, int* chosen_slots, int* chosen_tiles, double* best_ms,
                         cudaStream_t stream) {
  if (what != SB_TUNE_EVALUATE && what != SB_TUNE_MINIMIZE) {
    throw Error(SB_ERR_ARGUMENT, "autotune target must be SB_TUNE_EVALUATE or SB_TUNE_MINIMIZE");
  }
  if (fp64) {
    throw Error(SB_ERR_UNSUPPORTED, "the FP64 mode has no work-unit packing to tune");
  }
  static const int kFixed[][2] = {{256, 36}, {256, 24}, {192, 21}, {160, 15}, {128, 16},
                                  {128, 10}, {96, 12}, {96, 6}, {64, 6}, {256, 4}, {256, 1}};
  std::vector<std::pair<int, int>> candidates;
  for (const auto &c : kFixed) {
    candidates.emplace_back(c[0], c[1]);
  }
  if (what == SB_TUNE_EVALUATE) {
    // Wave-sized packings: tile caps that split the fused tiles into one to four waves of the
    // evaluation kernel's resident blocks (four per SM), so the last wave is not a sliver
    long long tiles_all = 0;
    for (int s = 0; s < nsys; s++) {
      if (atom_count[s] <= tiled_threshold) {
        const long long nb = (atom_count[s] + kTile - 1) / kTile;
        tiles_all += nb * (nb + 1) / 2;
      }
    }
    const long long resident = 4LL * sm_count;
    for (int waves = 1; waves <= 4; waves++) {
      const long long cap = (tiles_all + waves * resident - 1) / (waves * resident);
      if (cap >= 6 && cap <= 64) {
        const std::pair<int, int> c(256, static_cast<int>(cap));
        if (std::find(candidates.begin(), candidates.end(), c) == candidates.end()) {
          candidates.push_back(c);
        }
      }
    }
  }
  cudaEvent_t e0, e1;
  cudaCheck(cudaEventCreate(&e0), "cudaEventCreate");
  cudaCheck(cudaEventCreate(&e1), "cudaEventCreate");
  // the minimizer moves coordinates: keep a copy to restore between candidates
  const size_t np = natom_padded;
  DeviceArray<long long> keep;
  auto copy3 = [&](long long* dx, long long* dy, long long* dz, const long long* sx,
                   const long long* sy, const long long* sz) {
    cudaCheck(cudaMemcpyAsync(dx, sx, np * 8, cudaMemcpyDeviceToDevice, stream), "copy");
    cudaCheck(cudaMemcpyAsync(dy, sy, np * 8, cudaMemcpyDeviceToDevice, stream), "copy");
    cudaCheck(cudaMemcpyAsync(dz, sz, np * 8, cudaMemcpyDeviceToDevice, stream), "copy");
  };
  if (what == SB_TUNE_MINIMIZE) {
    keep.allocate(3 * np);
    copy3(keep.p, keep.p + np, keep.p + 2 * np, d_xcrd.p, d_ycrd.p, d_zcrd.p);
  }
  sb_minimize_controls ctl;
  sb_default_minimize_controls(&ctl);
  ctl.total_cycles = 8;
  ctl.sd_cycles = 4;
  double best = 1.0e30;
  std::unique_ptr<UnitPlan> best_plan;
  bool best_wide = allow_wide;
  const bool keep_wide = allow_wide;
  for (const auto &c : candidates) {
    std::unique_ptr<UnitPlan> plan;
    try {
      plan = makePlan(c.first, c.second);
    }
    catch (const Error &) {
      continue;   // a candidate that does not fit this synthesis
    }
    // evaluation packings are timed with both block-size rules: 512-thread blocks for launches
    // of fewer units than one wave of 256-thread blocks, or 256 threads throughout
    const int modes = (what == SB_TUNE_EVALUATE && opt.threads_per_block <= 0) ? 2 : 1;
    double plan_best = 1.0e30;
    bool plan_wide = keep_wide;
    for (int mode = 0; mode < modes; mode++) {
      allow_wide = (modes == 2) ? (mode == 0) : keep_wide;
      float ms = 0.0f;
      if (what == SB_TUNE_EVALUATE) {
        launchPlan(*plan, SB_TERM_ALL, true, true, stream);
        cudaCheck(cudaEventRecord(e0, stream), "cudaEventRecord");
        for (int r = 0; r < 3; r++) {
          launchPlan(*plan, SB_TERM_ALL, true, true, stream);
        }
        cudaCheck(cudaEventRecord(e1, stream), "cudaEventRecord");
      }
      else {
        minimizeBegin(ctl, stream);
        cudaCheck(cudaEventRecord(e0, stream), "cudaEventRecord");
        launchMinPlan(*plan, ctl.total_cycles, false, stream);
        cudaCheck(cudaEventRecord(e1, stream), "cudaEventRecord");
        copy3(d_xcrd.p, d_ycrd.p, d_zcrd.p, keep.p, keep.p + np, keep.p + 2 * np);
      }
      cudaCheck(cudaEventSynchronize(e1), "cudaEventSynchronize");
      cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      if (ms < plan_best) {
        plan_best = ms;
        plan_wide = allow_wide;
      }
    }
    allow_wide = keep_wide;
    if (plan_best < best) {
      best = plan_best;
      best_plan = std::move(plan);
      best_wide = plan_wide;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (what == SB_TUNE_EVALUATE) {
    // the candidates' evaluations accumulated into forces and energies: clear them
    initialize(SB_INIT_FORCES | SB_INIT_ENERGIES | SB_INIT_GB_WORKSPACE, stream);
  }
  cudaCheck(cudaStreamSynchronize(stream), "autotune");
  if (!best_plan) {
    throw Error(SB_ERR_ARGUMENT, "no work-unit packing fits this synthesis");
  }
  if (chosen_slots) *chosen_slots = best_plan->max_slots_cap;
  if (chosen_tiles) *chosen_tiles = best_plan->max_tiles_cap;
  if (best_ms) *best_ms = best;
  if (what == SB_TUNE_EVALUATE) {
    allow_wide = best_wide;
    eval_plan = std::move(best_plan);
    dev.nunit = eval_plan->units.size();
    dev.unit_desc = eval_plan->d_units.p;
    dev.unit_meta = eval_plan->d_meta.p;
  }
  else {
    min_plan = std::move(best_plan);
    min_ready = false;
  }
}

void Synthesis::getMinimizeHistory(double* out, cudaStream_t stream) {
  if (history_stride == 0) {
    throw Error(SB_ERR_ARGUMENT, "the last minimization kept no history");
  }
  cudaCheck(cudaMemcpyAsync(out, d_history.p,
                            sizeof(double) * static_cast<size_t>(nsys) * history_stride,
                            cudaMemcpyDeviceToHost, stream), "history download");
  cudaCheck(cudaStreamSynchronize(stream), "history download");
}

void Synthesis::getMinimizeProgress(int* cycles, int* converged, double* rms,
                                    cudaStream_t stream) {
  if (d_mcycle.p == nullptr) {
    throw Error(SB_ERR_ARGUMENT, "no minimization has run");
  }
  if (cycles) {
    cudaCheck(cudaMemcpyAsync(cycles, d_mcycle.p, sizeof(int) * nsys, cudaMemcpyDeviceToHost,
                              stream), "progress download");
  }
  if (converged) {
    cudaCheck(cudaMemcpyAsync(converged, d_mdone.p, sizeof(int) * nsys, cudaMemcpyDeviceToHost,
                              stream), "progress download");
  }
  if (rms) {
    cudaCheck(cudaMemcpyAsync(rms, d_rmsf.p, sizeof(double) * nsys, cudaMemcpyDeviceToHost,
                              stream), "progress download");
  }
  cudaCheck(cudaStreamSynchronize(stream), "progress download");
}

void Synthesis::exportMinimizerState(int system, MinimizerState* st, cudaStream_t stream) {
  if (!min_ready || fp64 || system < 0 || system >= nsys) {
    throw Error(SB_ERR_ARGUMENT, "minimizer state export needs a begun FP32 minimization and a "
                "system in range");
  }
  const int n = atom_count[system];
  const size_t a0 = atom_start[system];
  st->natom = n;
  const long long* crd[3] = {d_xcrd.p, d_ycrd.p, d_zcrd.p};
  const int* ovrf[3] = {d_xcrd_ovrf.p, d_ycrd_ovrf.p, d_zcrd_ovrf.p};
  const long long* prv[3] = {d_xprv.p, d_yprv.p, d_zprv.p};
  const float* cg[3] = {d_xcg.p, d_ycg.p, d_zcg.p};
  for (int c = 0; c < 3; c++) {
    st->crd[c].resize(n);
    st->crd_ovrf[c].resize(n);
    st->prv[c].resize(n);
    st->cg[c].resize(n);
    cudaCheck(cudaMemcpyAsync(st->crd[c].data(), crd[c] + a0, sizeof(long long) * n,
                              cudaMemcpyDeviceToHost, stream), "state export");
    cudaCheck(cudaMemcpyAsync(st->crd_ovrf[c].data(), ovrf[c] + a0, sizeof(int) * n,
                              cudaMemcpyDeviceToHost, stream), "state export");
    cudaCheck(cudaMemcpyAsync(st->prv[c].data(), prv[c] + a0, sizeof(long long) * n,
                              cudaMemcpyDeviceToHost, stream), "state export");
    cudaCheck(cudaMemcpyAsync(st->cg[c].data(), cg[c] + a0, sizeof(float) * n,
                              cudaMemcpyDeviceToHost, stream), "state export");
  }
  cudaCheck(cudaMemcpyAsync(&st->l_move, d_lmove.p + system, sizeof(double),
                            cudaMemcpyDeviceToHost, stream), "state export");
  cudaCheck(cudaMemcpyAsync(&st->rms_force, d_rmsf.p + system, sizeof(double),
                            cudaMemcpyDeviceToHost, stream), "state export");
  cudaCheck(cudaMemcpyAsync(&st->cycle, d_mcycle.p + system, sizeof(int),
                            cudaMemcpyDeviceToHost, stream), "state export");
  cudaCheck(cudaMemcpyAsync(&st->done, d_mdone.p + system, sizeof(int), cudaMemcpyDeviceToHost,
                            stream), "state export");
  cudaCheck(cudaStreamSynchronize(stream), "state export");
}

void Synthesis::importMinimizerState(int system, const MinimizerState &st,
                                     cudaStream_t stream) {
  if (!min_ready || fp64 || system < 0 || system >= nsys || st.natom != atom_count[system]) {
    throw Error(SB_ERR_ARGUMENT, "minimizer state import needs a begun FP32 minimization and a "
                "system of the same atom count");
  }
  const int n = st.natom;
  const size_t a0 = atom_start[system];
  long long* crd[3] = {d_xcrd.p, d_ycrd.p, d_zcrd.p};
  int* ovrf[3] = {d_xcrd_ovrf.p, d_ycrd_ovrf.p, d_zcrd_ovrf.p};
  long long* prv[3] = {d_xprv.p, d_yprv.p, d_zprv.p};
  float* cg[3] = {d_xcg.p, d_ycg.p, d_zcg.p};
  for (int c = 0; c < 3; c++) {
    cudaCheck(cudaMemcpyAsync(crd[c] + a0, st.crd[c].data(), sizeof(long long) * n,
                              cudaMemcpyHostToDevice, stream), "state import");
    cudaCheck(cudaMemcpyAsync(ovrf[c] + a0, st.crd_ovrf[c].data(), sizeof(int) * n,
                              cudaMemcpyHostToDevice, stream), "state import");
    cudaCheck(cudaMemcpyAsync(prv[c] + a0, st.prv[c].data(), sizeof(long long) * n,
                              cudaMemcpyHostToDevice, stream), "state import");
    cudaCheck(cudaMemcpyAsync(cg[c] + a0, st.cg[c].data(), sizeof(float) * n,
                              cudaMemcpyHostToDevice, stream), "state import");
  }
  cudaCheck(cudaMemcpyAsync(d_lmove.p + system, &st.l_move, sizeof(double),
                            cudaMemcpyHostToDevice, stream), "state import");
  cudaCheck(cudaMemcpyAsync(d_rmsf.p + system, &st.rms_force, sizeof(double),
                            cudaMemcpyHostToDevice, stream), "state import");
  cudaCheck(cudaMemcpyAsync(d_mcycle.p + system, &st.cycle, sizeof(int),
                            cudaMemcpyHostToDevice, stream), "state import");
  cudaCheck(cudaMemcpyAsync(d_mdone.p + system, &st.done, sizeof(int), cudaMemcpyHostToDevice,
                            stream), "state import");
  // the host copies are the caller's: wait until they have been read
  cudaCheck(cudaStreamSynchronize(stream), "state import");
}

}  // namespace sb

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
struct sb_synthesis {
  std::unique_ptr<sb::Synthesis> impl;
};

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

cudaStream_t asStream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

sb::Synthesis* need(sb_synthesis* syn) {
  if (syn == nullptr || !syn->impl) {
    throw sb::Error(SB_ERR_ARGUMENT, "null synthesis handle");
  }
  return syn->impl.get();
}

const sb::Synthesis* need(const sb_synthesis* syn) {
  if (syn == nullptr || !syn->impl) {
    throw sb::Error(SB_ERR_ARGUMENT, "null synthesis handle");
  }
  return syn->impl.get();
}

}  // namespace

extern "C" {

void sb_default_options(sb_options* opt) {
  std::memset(opt, 0, sizeof(sb_options));
  opt->igb = SB_GB_OBC2;
  opt->dielectric = 80.0;
  opt->saltcon = 0.0;
  opt->coulomb_constant = 332.0522172900000;
  opt->gpos_bits = 32;
  opt->frc_bits = 23;
  opt->nrg_bits = 26;
  opt->device = 0;
}

int sb_synthesis_create(const sb_topology* tops, int ntop, const int* topology_index, int nsys,
                        const sb_options* opt, sb_synthesis** out) {
  return guarded([&]() {
    if (out == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    sb_options o;
    if (opt != nullptr) {
      o = *opt;
    }
    else {
      sb_default_options(&o);
    }
    auto h = std::make_unique<sb_synthesis>();
    h->impl = std::make_unique<sb::Synthesis>(tops, ntop, topology_index, nsys, o);
    *out = h.release();
  });
}

int sb_synthesis_destroy(sb_synthesis* syn) {
  return guarded([&]() { delete syn; });
}

int sb_system_count(const sb_synthesis* syn) {
  if (syn == nullptr || !syn->impl) return SB_ERR_ARGUMENT;
  return syn->impl->nsys;
}

int sb_system_atoms(const sb_synthesis* syn, int system, int* natom, int* offset) {
  return guarded([&]() {
    const sb::Synthesis* s = need(syn);
    if (system < 0 || system >= s->nsys) throw sb::Error(SB_ERR_ARGUMENT, "system out of range");
    if (natom) *natom = s->atom_count[system];
    if (offset) *offset = s->atom_start[system];
  });
}

int sb_padded_atom_count(const sb_synthesis* syn) {
  if (syn == nullptr || !syn->impl) return SB_ERR_ARGUMENT;
  return syn->impl->natom_padded;
}

int sb_set_coordinates(sb_synthesis* syn, const double* xyz, void* stream) {
  return guarded([&]() { need(syn)->setCoordinates(xyz, asStream(stream)); });
}

int sb_get_coordinates(sb_synthesis* syn, double* xyz, void* stream) {
  return guarded([&]() { need(syn)->getCoordinates(xyz, asStream(stream)); });
}

int sb_get_forces(sb_synthesis* syn, double* xyz, void* stream) {
  return guarded([&]() { need(syn)->getForces(xyz, asStream(stream)); });
}

int sb_get_energies(sb_synthesis* syn, double* energies, void* stream) {
  return guarded([&]() { need(syn)->getEnergies(energies, asStream(stream)); });
}

int sb_set_restraints(sb_synthesis* syn, const sb_restraint* restraints, int count) {
  return guarded([&]() { need(syn)->setRestraints(restraints, count); });
}

int sb_surface_area(sb_synthesis* syn, const double* sphere_points, int n_points,
                    double probe_radius, double weight, double* out, void* stream) {
  return guarded([&]() {
    need(syn)->surfaceArea(sphere_points, n_points, probe_radius, weight, out, asStream(stream));
  });
}

int sb_set_restraint_step(sb_synthesis* syn, int step) {
  return guarded([&]() {
    if (step < 0) throw sb::Error(SB_ERR_ARGUMENT, "restraint step must be non-negative");
    need(syn)->dev_charmm.rst_step = step;
  });
}

int sb_download_results_async(sb_synthesis* syn, double* forces, double* energies,
                              void* stream) {
  return guarded([&]() { need(syn)->downloadResults(forces, energies, asStream(stream)); });
}

int sb_get_gb_workspace(sb_synthesis* syn, double* psi, double* radii, double* sumdeijda,
                        void* stream) {
  return guarded([&]() { need(syn)->getGbWorkspace(psi, radii, sumdeijda, asStream(stream)); });
}

int sb_get_forces_fixed(sb_synthesis* syn, int64_t* xyz_primary, int32_t* xyz_overflow,
                        void* stream) {
  return guarded([&]() {
    need(syn)->getForcesFixed(reinterpret_cast<long long*>(xyz_primary),
                              reinterpret_cast<int*>(xyz_overflow), asStream(stream));
  });
}

int sb_get_energies_fixed(sb_synthesis* syn, int64_t* energies, void* stream) {
  return guarded([&]() {
    need(syn)->getEnergiesFixed(reinterpret_cast<long long*>(energies), asStream(stream));
  });
}

int sb_initialize(sb_synthesis* syn, int what, void* stream) {
  return guarded([&]() { need(syn)->initialize(what, asStream(stream)); });
}

int sb_evaluate(sb_synthesis* syn, int terms, int eval_force, int eval_energy, void* stream) {
  return guarded([&]() {
    need(syn)->evaluate(terms, eval_force != 0, eval_energy != 0, asStream(stream));
  });
}

int sb_evaluate_range(sb_synthesis* syn, int first, int count, int terms, int eval_force,
                      int eval_energy, void* stream) {
  return guarded([&]() {
    need(syn)->evaluateRange(first, count, terms, eval_force != 0, eval_energy != 0,
                             asStream(stream));
  });
}

int sb_evaluate_clash(sb_synthesis* syn, int terms, int eval_force, int eval_energy,
                      double clash_distance, double clash_ratio, void* stream) {
  return guarded([&]() {
    if (!(clash_distance >= 0.0) || !(clash_ratio >= 0.0) || !std::isfinite(clash_distance) ||
        !std::isfinite(clash_ratio)) {
      throw sb::Error(SB_ERR_ARGUMENT, "clash distance and ratio must be finite, not negative");
    }
    sb::Clash clash;
    clash.distance = static_cast<float>(clash_distance);
    clash.ratio = static_cast<float>(clash_ratio);
    clash.distance64 = clash_distance;
    clash.ratio64 = clash_ratio;
    need(syn)->evaluate(terms, eval_force != 0, eval_energy != 0, asStream(stream), clash);
  });
}

int sb_launch_nonbonded(sb_synthesis* syn, int eval_force, int eval_energy, void* stream) {
  return guarded([&]() {
    need(syn)->evaluate(SB_TERM_NONBONDED | SB_TERM_GB, eval_force != 0, eval_energy != 0,
                        asStream(stream));
  });
}

int sb_launch_valence(sb_synthesis* syn, int eval_force, int eval_energy, void* stream) {
  return guarded([&]() {
    need(syn)->evaluate(SB_TERM_VALENCE, eval_force != 0, eval_energy != 0, asStream(stream));
  });
}

int sb_launch_info(const sb_synthesis* syn, int* work_units, int* blocks, int* threads) {
  return guarded([&]() {
    const sb::Synthesis* s = need(syn);
    if (work_units) *work_units = s->eval_plan->units.size();
    if (blocks) *blocks = s->eval_plan->units.size();
    if (threads) {
      // block size of the batched evaluation's launch of packed units
      const int n = static_cast<int>(s->eval_plan->units.size());
      const int packed = n - s->eval_plan->n_big;
      *threads = s->launchThreads(packed > 0 ? packed : n, SB_TERM_ALL);
    }
  });
}

int sb_check_status(sb_synthesis* syn, int* status) {
  return guarded([&]() {
    const int st = need(syn)->checkStatus(nullptr);
    if (status) *status = st;
  });
}

void sb_default_minimize_controls(sb_minimize_controls* ctl) {
  std::memset(ctl, 0, sizeof(sb_minimize_controls));
  ctl->kernel = SB_MIN_GRAPH;
  ctl->total_cycles = 200;
  ctl->sd_cycles = 50;
  ctl->clash_cycles = 0;
  ctl->clash_distance = 0.2;
  ctl->clash_ratio = 0.5;
  ctl->initial_step = 0.01;
  ctl->convergence_rms = 0.0;
  ctl->record_history = 0;
}

int sb_minimize(sb_synthesis* syn, const sb_minimize_controls* ctl, void* stream) {
  return guarded([&]() {
    if (ctl == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null minimization controls");
    need(syn)->minimize(*ctl, asStream(stream));
  });
}

int sb_minimize_range(sb_synthesis* syn, int first, int count, const sb_minimize_controls* ctl,
                      void* stream) {
  return guarded([&]() {
    if (ctl == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null minimization controls");
    need(syn)->minimizeRange(first, count, *ctl, asStream(stream));
  });
}

int sb_minimize_begin(sb_synthesis* syn, const sb_minimize_controls* ctl, void* stream) {
  return guarded([&]() {
    if (ctl == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null minimization controls");
    need(syn)->minimizeBegin(*ctl, asStream(stream));
  });
}

int sb_minimize_advance(sb_synthesis* syn, int cycles, int final_energy, void* stream) {
  return guarded([&]() {
    need(syn)->minimizeAdvance(cycles, final_energy != 0, asStream(stream));
  });
}

int sb_conjugate_gradient(sb_synthesis* syn, void* stream) {
  return guarded([&]() { need(syn)->conjugateGradient(asStream(stream)); });
}

int sb_line_advance(sb_synthesis* syn, int move_number, void* stream) {
  return guarded([&]() { need(syn)->lineAdvance(move_number, asStream(stream)); });
}

int sb_autotune(sb_synthesis* syn, int what, int* max_atoms_per_unit, int* max_tiles_per_unit,
                double* best_ms, void* stream) {
  return guarded([&]() {
    need(syn)->autotune(what, max_atoms_per_unit, max_tiles_per_unit, best_ms, asStream(stream));
  });
}

int sb_get_minimize_history(sb_synthesis* syn, double* history, void* stream) {
  return guarded([&]() {
    if (history == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null output");
    need(syn)->getMinimizeHistory(history, asStream(stream));
  });
}

int sb_get_minimize_progress(sb_synthesis* syn, int* cycles_done, int* converged,
                             double* rms_force, void* stream) {
  return guarded([&]() {
    need(syn)->getMinimizeProgress(cycles_done, converged, rms_force, asStream(stream));
  });
}

const char* sb_last_error(void) { return sb::lastError(); }

const char* sb_version(void) { return "stormm_b200 0.1 (sm_100a)"; }

}  // extern "C"
