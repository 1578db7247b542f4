/*
 * stormm_b200.hpp: STORMM's C++ classes and launchers for this path, header only, over the C
 * ABI of stormm_b200.h.
 *
 * A caller written against STORMM's API (namespace stormm) compiles against this header with the
 * same class names, constructor arguments, launcher signatures and argument meanings, and the
 * same error behaviour (std::runtime_error, as STORMM's rtErr throws):
 *
 *   AtomGraph ag("molecule.prmtop");                       Topology/atomgraph.h:83,156
 *   PhaseSpace ps("molecule.inpcrd");                      Trajectory/phasespace.h
 *   AtomGraphSynthesis poly_ag({&ag, ...}, {0, 0, ...});   Synthesis/atomgraph_synthesis.h:97-100
 *   poly_ag.setImplicitSolventModel(ImplicitSolventModel::OBC_GB_II);
 *   PhaseSpaceSynthesis poly_ps({ps, ...}, {&ag, ...});    Synthesis/phasespace_synthesis.h:348
 *   StaticExclusionMaskSynthesis poly_se(poly_ag);
 *   poly_ag.upload();  poly_ps.upload();
 *   ScoreCard sc(poly_ag.getSystemCount());
 *   ImplicitSolventWorkspace ism_space(poly_ag);
 *   launchNonbonded(PrecisionModel::SINGLE, poly_ag, poly_se, &mmctrl, &poly_ps, &heat_bath,
 *                   &sc, &tb_space, &ism_space, EvaluateForce::YES, EvaluateEnergy::YES,
 *                   launcher);                             Potential/hpc_nonbonded_potential.h:142
 *   launchValence(PrecisionModel::SINGLE, poly_ag, &mmctrl, &poly_ps, &heat_bath, &sc,
 *                 &tb_space, EvaluateForce::YES, EvaluateEnergy::YES, VwuGoal::ACCUMULATE,
 *                 launcher);                               Potential/hpc_valence_potential.h:312
 *   ScoreCard e = launchMinimization(poly_ag, poly_se, &poly_ps, mincon, gpu);
 *                                                          MolecularMechanics/hpc_minimization.h:136
 *   sc.download();  poly_ps.download();
 *
 * Where the B200 design differs underneath:
 *   - One device object (sb_synthesis) holds topology, coordinates, forces, GB workspace and
 *     energies.  AtomGraphSynthesis::upload creates it; the PhaseSpaceSynthesis, ScoreCard and
 *     ImplicitSolventWorkspace given to a launcher are bound to that synthesis there, and their
 *     upload / initialize requests made before the binding are carried out at it.  Bind one
 *     PhaseSpaceSynthesis per AtomGraphSynthesis: binding another one uploads its coordinates
 *     over the first one's.
 *   - The precision model is chosen at upload (FP32 arithmetic with fixed-point accumulation,
 *     or FP64 arithmetic); a launch with the other model throws.  FP64 minimization runs the
 *     graph minimizer with the direction in FP64.
 *   - The GB model, dielectric and salt concentration are one per synthesis.
 *   - CacheResource, Thermostat, ReductionBridge, StopWatch and the AccumulationMethod argument
 *     are accepted and have nothing to carry: a thread block holds a whole work unit on chip,
 *     accumulation is always int64 + int32 overflow, and the minimizer keeps its line-search
 *     state on the device.  MolecularMechanicsControls carries the minimizer's cycle counts and
 *     move length to launchConjugateGradient; LineMinimization names the system count.  CoreKlManager
 *     carries the CUDA stream the launches go to (default stream unless set).
 *   - Streams are given as void* (cudaStream_t), so this header needs no CUDA header.
 */
#ifndef STORMM_B200_HPP
#define STORMM_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "stormm_b200.h"

namespace stormm_b200 {

/* ------------------------------------------------------------------------------------------ */
/* Enumerations, in STORMM's order                                                             */
/* ------------------------------------------------------------------------------------------ */
enum class PrecisionModel { SINGLE, DOUBLE };                      // Constants/behavior.h:32-37
enum class EvaluateForce { NO, YES };                              // Potential/energy_enumerators.h:19
enum class EvaluateEnergy { NO, YES };                             // Potential/energy_enumerators.h:14
enum class AccumulationMethod { SPLIT, WHOLE, AUTOMATIC };         // Numerics/numeric_enumerators.h:12
enum class VwuGoal { ACCUMULATE, MOVE_PARTICLES };                 // Synthesis/synthesis_enumerators.h:88
enum class ImplicitSolventModel {                                  // Topology/atomgraph_enumerators.h:141
  NONE, HCT_GB, OBC_GB, OBC_GB_II, NECK_GB, NECK_GB_II
};
enum class AtomicRadiusSet {                                       // Topology/atomgraph_enumerators.h:150
  NONE, BONDI, AMBER6, MBONDI, MBONDI2, MBONDI3, PARSE
};
enum class InitializationTask {                                    // Synthesis/synthesis_enumerators.h:109
  GENERAL_DYNAMICS, GB_DYNAMICS, GENERAL_MINIMIZATION, GB_MINIMIZATION, LANGEVIN_DYNAMICS,
  GB_LANGEVIN_DYNAMICS, NONE
};
enum class TrajectoryKind { POSITIONS, VELOCITIES, FORCES };      // Trajectory/trajectory_enumerators.h
enum class StateVariable {                                         // Potential/energy_enumerators.h:36-68
  BOND = 0, ANGLE, PROPER_DIHEDRAL, IMPROPER_DIHEDRAL, UREY_BRADLEY, CHARMM_IMPROPER, CMAP, VDW,
  VDW_ONE_FOUR, ELECTROSTATIC, ELEC_ONE_FOUR, GENERALIZED_BORN, RESTRAINT, SURFACE_AREA, KINETIC,
  PRESSURE, VIRIAL_11, VIRIAL_12, VIRIAL_22, VIRIAL_13, VIRIAL_23, VIRIAL_33, VOLUME,
  TEMPERATURE_ALL, TEMPERATURE_PROTEIN, TEMPERATURE_LIGAND, TEMPERATURE_SOLVENT, DU_DLAMBDA,
  POTENTIAL_ENERGY, TOTAL_ENERGY, ALL_STATES
};

constexpr int default_energy_scale_bits = 26;                      // Constants/fixed_precision.h:121

namespace detail {

inline void check(int rc, const std::string &where) {
  if (rc != SB_OK) {
    const char* msg = sb_last_error();
    throw std::runtime_error(where + ": " + (msg != nullptr ? msg : "error ") +
                             " (status " + std::to_string(rc) + ")");
  }
}

inline int igbNumber(ImplicitSolventModel m) {
  switch (m) {
  case ImplicitSolventModel::NONE: return SB_GB_NONE;
  case ImplicitSolventModel::HCT_GB: return SB_GB_HCT;
  case ImplicitSolventModel::OBC_GB: return SB_GB_OBC;
  case ImplicitSolventModel::OBC_GB_II: return SB_GB_OBC2;
  case ImplicitSolventModel::NECK_GB: return SB_GB_NECK;
  case ImplicitSolventModel::NECK_GB_II: return SB_GB_NECK2;
  }
  return SB_GB_NONE;
}

template <typename T> std::vector<T> copyOf(const T* p, size_t n) {
  return (p == nullptr || n == 0) ? std::vector<T>() : std::vector<T>(p, p + n);
}

template <typename T> const T* dataOrNull(const std::vector<T> &v) {
  return v.empty() ? nullptr : v.data();
}

}  // namespace detail

/* ------------------------------------------------------------------------------------------ */
/* Placeholders for STORMM objects whose role lives inside the library                         */
/* ------------------------------------------------------------------------------------------ */
class GpuDetails {                                                 // Accelerator/gpu_details.h
public:
  explicit GpuDetails(int device_index = 0) : device(device_index) {}
  int getDeviceIndex() const { return device; }
private:
  int device;
};

class MinimizeControls;
/* MolecularMechanicsControls (MolecularMechanics/mm_controls.h:100-140): for a minimization it
 * carries the cycle counts and the initial move length the line-search steps use
 * (launchConjugateGradient begins the synthesis' minimizer state from them on its first call).
 * STORMM's work-unit counters have no counterpart: a thread block holds a whole unit on chip. */
class MolecularMechanicsControls {
public:
  explicit MolecularMechanicsControls(double initial_step_in = 0.01)
      : initial_step(initial_step_in) {}
  explicit MolecularMechanicsControls(const MinimizeControls &user_input);
  int getTotalCycles() const { return total_cycles; }
  int getSteepestDescentCycles() const { return sd_cycles; }
  double getInitialStep() const { return initial_step; }
  /* The synthesis whose minimizer these controls began (nullptr: none yet) */
  const void* begunFor() const { return begun; }
  void markBegun(const void* handle) { begun = handle; }

private:
  int total_cycles = 200, sd_cycles = 50;
  double initial_step = 0.01;
  const void* begun = nullptr;
};
class Thermostat {};                                               // Trajectory/thermostat.h
class CacheResource {};                                            // Accelerator/cacheresource.h:63
class ReductionBridge {                                            // Math/reduction_bridge.h:24
public:
  explicit ReductionBridge(size_t = 0) {}
};
/* LineMinimization (MolecularMechanics/line_minimization.h:85-100): the per-system line-search
 * record lives on the device with the synthesis; this object names the system count */
class LineMinimization {
public:
  explicit LineMinimization(int system_count_in = 0, double dx0 = 0.0)
      : system_count(system_count_in), initial_step(dx0) {}
  int getSystemCount() const { return system_count; }
  double getInitialStep() const { return initial_step; }

private:
  int system_count;
  double initial_step;
};
class StopWatch {};                                                // UnitTesting/stopwatch.h

/* ------------------------------------------------------------------------------------------ */
/* Topologies and coordinates                                                                  */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's NeckGeneralizedBornTable (Potential/neck_gb_table.h): the caller supplies the
 * size x size maximum separations and values, indexed [j * size + i]. */
class NeckGeneralizedBornTable {
public:
  NeckGeneralizedBornTable(int table_size, std::vector<double> max_separation,
                           std::vector<double> max_value, double neck_cut = 6.8)
      : size(table_size), sep(std::move(max_separation)), val(std::move(max_value)),
        cut(neck_cut) {
    if (size <= 0 || sep.size() != static_cast<size_t>(size) * size ||
        val.size() != sep.size()) {
      throw std::runtime_error("NeckGeneralizedBornTable: tables must hold size^2 values");
    }
  }
  int getTableSize() const { return size; }
  const std::vector<double> &getMaxSeparation() const { return sep; }
  const std::vector<double> &getMaxValue() const { return val; }
  double getNeckCut() const { return cut; }
private:
  int size;
  std::vector<double> sep, val;
  double cut;
};

/* One molecule's topology.  Read from an Amber prmtop (STORMM's AtomGraph(file_name)) or copied
 * from an sb_topology a caller filled. */
class AtomGraph {
public:
  explicit AtomGraph(const std::string &file_name) : source(file_name) {
    sb_amber_topology* h = nullptr;
    detail::check(sb_read_amber_topology(file_name.c_str(), &h), "AtomGraph");
    amber.reset(h, [](sb_amber_topology* p) { sb_amber_topology_destroy(p); });
    refreshFromFile();
  }

  explicit AtomGraph(const sb_topology &top) : source("(arrays)") { copyTopology(top); }

  int getAtomCount() const { return view.natom; }
  const std::string &getFileName() const { return source; }
  const std::vector<int> &getAtomicNumbers() const { return z_numbers; }
  int getCmapTermCount() const { return cmap_count; }

  /* STORMM's AtomGraph::setImplicitSolventModel (Topology/atomgraph_setters.cpp:672-1060).  For
   * a topology read from a file: the radius set, element screening factors of the neck models
   * and per-model alpha / beta / gamma, as STORMM assigns them.  For a topology given as arrays:
   * the model, dielectric and salt are recorded; its radii, screening factors and alpha / beta /
   * gamma (NULL: the model's uniform values) are kept. */
  void setImplicitSolventModel(ImplicitSolventModel igb_in, double dielectric_in = 80.0,
                               double saltcon_in = 0.0,
                               AtomicRadiusSet radii_set = AtomicRadiusSet::NONE) {
    if (amber) {
      detail::check(sb_amber_set_implicit_solvent(amber.get(), detail::igbNumber(igb_in),
                                                  static_cast<int>(radii_set)),
                    "AtomGraph::setImplicitSolventModel");
      refreshFromFile();
    }
    else if (radii_set != AtomicRadiusSet::NONE) {
      throw std::runtime_error("AtomGraph::setImplicitSolventModel: a radius set needs a "
                               "topology read from a file (atom names, elements, residues)");
    }
    gb_model = igb_in;
    dielectric = dielectric_in;
    saltcon = saltcon_in;
    model_set = true;
  }
  ImplicitSolventModel getImplicitSolventModel() const { return gb_model; }
  double getDielectricConstant() const { return dielectric; }
  double getSaltConcentration() const { return saltcon; }
  bool implicitSolventModelSet() const { return model_set; }

  /* The topology in the C ABI's form; pointers stay valid while this AtomGraph lives and its
   * solvent model is not changed */
  const sb_topology &abi() const { return view; }

private:
  std::string source;
  std::shared_ptr<sb_amber_topology> amber;
  sb_topology view{};
  std::vector<double> charge, lja, ljb, lja14, ljb14, radii, screen, alpha, beta, gamma;
  std::vector<double> bond_k, bond_r, angl_k, angl_t, dihe_amp, dihe_freq, dihe_phase;
  std::vector<double> dihe_scee, dihe_scnb;
  std::vector<int> lj_idx, excl_bounds, excl_list, bonds, angles, dihedrals, improper;
  std::vector<int> z_numbers;
  int cmap_count = 0;
  ImplicitSolventModel gb_model = ImplicitSolventModel::NONE;
  double dielectric = 80.0, saltcon = 0.0;
  bool model_set = false;

  void refreshFromFile() {
    sb_amber_view v;
    detail::check(sb_amber_topology_view(amber.get(), &v), "AtomGraph");
    copyTopology(v.topology);
    z_numbers = detail::copyOf(v.atomic_numbers, static_cast<size_t>(v.topology.natom));
    cmap_count = v.cmap_count;
  }

  void copyTopology(const sb_topology &t) {
    if (t.natom <= 0 || t.excl_bounds == nullptr) {
      throw std::runtime_error("AtomGraph: a topology needs atoms and exclusion bounds");
    }
    const size_t n = static_cast<size_t>(t.natom);
    const size_t nt2 = static_cast<size_t>(t.n_lj_types) * t.n_lj_types;
    charge = detail::copyOf(t.charge, n);
    lj_idx = detail::copyOf(t.lj_idx, n);
    lja = detail::copyOf(t.lja, nt2);
    ljb = detail::copyOf(t.ljb, nt2);
    lja14 = detail::copyOf(t.lja14, nt2);
    ljb14 = detail::copyOf(t.ljb14, nt2);
    excl_bounds = detail::copyOf(t.excl_bounds, n + 1);
    excl_list = detail::copyOf(t.excl_list, static_cast<size_t>(t.excl_bounds[n]));
    radii = detail::copyOf(t.pb_radii, n);
    screen = detail::copyOf(t.gb_screen, n);
    alpha = detail::copyOf(t.gb_alpha, n);
    beta = detail::copyOf(t.gb_beta, n);
    gamma = detail::copyOf(t.gb_gamma, n);
    bonds = detail::copyOf(t.bond_atoms, 2 * static_cast<size_t>(t.nbond));
    bond_k = detail::copyOf(t.bond_keq, static_cast<size_t>(t.nbond));
    bond_r = detail::copyOf(t.bond_leq, static_cast<size_t>(t.nbond));
    angles = detail::copyOf(t.angl_atoms, 3 * static_cast<size_t>(t.nangl));
    angl_k = detail::copyOf(t.angl_keq, static_cast<size_t>(t.nangl));
    angl_t = detail::copyOf(t.angl_theta0, static_cast<size_t>(t.nangl));
    dihedrals = detail::copyOf(t.dihe_atoms, 4 * static_cast<size_t>(t.ndihe));
    dihe_amp = detail::copyOf(t.dihe_amp, static_cast<size_t>(t.ndihe));
    dihe_freq = detail::copyOf(t.dihe_freq, static_cast<size_t>(t.ndihe));
    dihe_phase = detail::copyOf(t.dihe_phase, static_cast<size_t>(t.ndihe));
    dihe_scee = detail::copyOf(t.dihe_scee, static_cast<size_t>(t.ndihe));
    dihe_scnb = detail::copyOf(t.dihe_scnb, static_cast<size_t>(t.ndihe));
    improper = detail::copyOf(t.dihe_improper, static_cast<size_t>(t.ndihe));
    view = t;
    view.charge = detail::dataOrNull(charge);
    view.lj_idx = detail::dataOrNull(lj_idx);
    view.lja = detail::dataOrNull(lja);
    view.ljb = detail::dataOrNull(ljb);
    view.lja14 = detail::dataOrNull(lja14);
    view.ljb14 = detail::dataOrNull(ljb14);
    view.excl_bounds = detail::dataOrNull(excl_bounds);
    view.excl_list = detail::dataOrNull(excl_list);
    view.pb_radii = detail::dataOrNull(radii);
    view.gb_screen = detail::dataOrNull(screen);
    view.gb_alpha = detail::dataOrNull(alpha);
    view.gb_beta = detail::dataOrNull(beta);
    view.gb_gamma = detail::dataOrNull(gamma);
    view.bond_atoms = detail::dataOrNull(bonds);
    view.bond_keq = detail::dataOrNull(bond_k);
    view.bond_leq = detail::dataOrNull(bond_r);
    view.angl_atoms = detail::dataOrNull(angles);
    view.angl_keq = detail::dataOrNull(angl_k);
    view.angl_theta0 = detail::dataOrNull(angl_t);
    view.dihe_atoms = detail::dataOrNull(dihedrals);
    view.dihe_amp = detail::dataOrNull(dihe_amp);
    view.dihe_freq = detail::dataOrNull(dihe_freq);
    view.dihe_phase = detail::dataOrNull(dihe_phase);
    view.dihe_scee = detail::dataOrNull(dihe_scee);
    view.dihe_scnb = detail::dataOrNull(dihe_scnb);
    view.dihe_improper = detail::dataOrNull(improper);
  }
};

/* One system's coordinates and forces (host memory, interlaced x, y, z), STORMM's PhaseSpace */
class PhaseSpace {
public:
  explicit PhaseSpace(int atom_count = 0)
      : natom(atom_count), xyz(3 * static_cast<size_t>(atom_count), 0.0),
        frc(3 * static_cast<size_t>(atom_count), 0.0) {}

  /* Amber ASCII coordinate or restart file */
  explicit PhaseSpace(const std::string &file_name) {
    std::ifstream in(file_name);
    std::string title, counts;
    if (!in || !std::getline(in, title) || !std::getline(in, counts)) {
      throw std::runtime_error("PhaseSpace: cannot read coordinate file " + file_name);
    }
    std::istringstream ss(counts);
    if (!(ss >> natom) || natom <= 0) {
      throw std::runtime_error("PhaseSpace: no atom count in " + file_name);
    }
    xyz.assign(3 * static_cast<size_t>(natom), 0.0);
    frc.assign(xyz.size(), 0.0);
    detail::check(sb_read_amber_coordinates(file_name.c_str(), natom, xyz.data()), "PhaseSpace");
  }

  PhaseSpace(int atom_count, const std::vector<double> &interlaced_xyz) : PhaseSpace(atom_count) {
    if (interlaced_xyz.size() != xyz.size()) {
      throw std::runtime_error("PhaseSpace: coordinate array does not match the atom count");
    }
    xyz = interlaced_xyz;
  }

  int getAtomCount() const { return natom; }
  std::vector<double> getInterlacedCoordinates(
      TrajectoryKind kind = TrajectoryKind::POSITIONS) const {
    switch (kind) {
    case TrajectoryKind::POSITIONS: return xyz;
    case TrajectoryKind::FORCES: return frc;
    case TrajectoryKind::VELOCITIES: return std::vector<double>(xyz.size(), 0.0);
    }
    return xyz;
  }

private:
  friend class PhaseSpaceSynthesis;
  int natom = 0;
  std::vector<double> xyz, frc;
};

class AtomGraphSynthesis;

/* ------------------------------------------------------------------------------------------ */
/* Syntheses                                                                                   */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's AtomGraphSynthesis: the topologies of every system.  upload() builds the device
 * synthesis that also holds coordinates, forces, GB workspace and energies. */
class AtomGraphSynthesis {
public:
  AtomGraphSynthesis(const std::vector<AtomGraph*> &topologies_in,
                     const std::vector<int> &topology_indices_in)
      : topologies(topologies_in), indices(topology_indices_in) {
    if (topologies.empty() || indices.empty()) {
      throw std::runtime_error("AtomGraphSynthesis: no topologies or no systems");
    }
    for (AtomGraph* ag : topologies) {
      if (ag == nullptr) {
        throw std::runtime_error("AtomGraphSynthesis: null topology");
      }
    }
    for (int k : indices) {
      if (k < 0 || k >= static_cast<int>(topologies.size())) {
        throw std::runtime_error("AtomGraphSynthesis: topology index " + std::to_string(k) +
                                 " out of range");
      }
    }
    sb_default_options(&opt);
    // A model already set on the topologies becomes the synthesis' (all must agree)
    const AtomGraph* first = topologies[0];
    if (first->implicitSolventModelSet()) {
      for (AtomGraph* ag : topologies) {
        if (!ag->implicitSolventModelSet() ||
            ag->getImplicitSolventModel() != first->getImplicitSolventModel() ||
            ag->getDielectricConstant() != first->getDielectricConstant() ||
            ag->getSaltConcentration() != first->getSaltConcentration()) {
          throw std::runtime_error("AtomGraphSynthesis: topologies with different implicit "
                                   "solvent models");
        }
      }
      model = first->getImplicitSolventModel();
      opt.igb = detail::igbNumber(model);
      opt.dielectric = first->getDielectricConstant();
      opt.saltcon = first->getSaltConcentration();
    }
  }

  explicit AtomGraphSynthesis(const std::vector<AtomGraph*> &topologies_in)
      : AtomGraphSynthesis(topologies_in, identity(topologies_in.size())) {}

  AtomGraphSynthesis(const AtomGraphSynthesis &) = delete;
  AtomGraphSynthesis &operator=(const AtomGraphSynthesis &) = delete;
  ~AtomGraphSynthesis() {
    if (syn != nullptr) {
      sb_synthesis_destroy(syn);
    }
  }

  /* STORMM's AtomGraphSynthesis::setImplicitSolventModel (atomgraph_synthesis.h:440-473): sets
   * the model on every topology, then on the synthesis.  Before upload() only. */
  void setImplicitSolventModel(ImplicitSolventModel igb_in,
                               AtomicRadiusSet radii_set = AtomicRadiusSet::NONE,
                               double dielectric_in = 80.0, double saltcon_in = 0.0) {
    if (igb_in == ImplicitSolventModel::NECK_GB || igb_in == ImplicitSolventModel::NECK_GB_II) {
      throw std::runtime_error("AtomGraphSynthesis::setImplicitSolventModel: the neck models "
                               "need a NeckGeneralizedBornTable");
    }
    applyModel(igb_in, radii_set, dielectric_in, saltcon_in);
  }

  void setImplicitSolventModel(ImplicitSolventModel igb_in,
                               const NeckGeneralizedBornTable &ngb_tab,
                               AtomicRadiusSet radii_set = AtomicRadiusSet::NONE,
                               double dielectric_in = 80.0, double saltcon_in = 0.0) {
    neck_sep = ngb_tab.getMaxSeparation();
    neck_val = ngb_tab.getMaxValue();
    opt.neck_table_size = ngb_tab.getTableSize();
    opt.neck_cut = ngb_tab.getNeckCut();
    applyModel(igb_in, radii_set, dielectric_in, saltcon_in);
  }

  ImplicitSolventModel getImplicitSolventModel() const { return model; }
  int getSystemCount() const { return static_cast<int>(indices.size()); }
  int getAtomCount(int system) const {
    return topologies.at(static_cast<size_t>(indices.at(static_cast<size_t>(system))))
        ->getAtomCount();
  }
  const std::vector<int> &getTopologyIndices() const { return indices; }
  const std::vector<AtomGraph*> &getUniqueTopologies() const { return topologies; }
  int getEnergyScaleBits() const { return opt.nrg_bits; }

  /* Further options of the C ABI (work-unit packing, fixed-point bits, device) before upload */
  sb_options &options() {
    requireNotUploaded("options");
    return opt;
  }

  /* Build the device synthesis with the chosen precision model */
  void upload(PrecisionModel prec = PrecisionModel::SINGLE) {
    requireNotUploaded("upload");
    std::vector<sb_topology> tops;
    tops.reserve(topologies.size());
    for (AtomGraph* ag : topologies) {
      tops.push_back(ag->abi());
    }
    opt.precision = (prec == PrecisionModel::DOUBLE) ? SB_PRECISION_DOUBLE : SB_PRECISION_SINGLE;
    opt.neck_max_separation = detail::dataOrNull(neck_sep);
    opt.neck_max_value = detail::dataOrNull(neck_val);
    detail::check(sb_synthesis_create(tops.data(), static_cast<int>(tops.size()), indices.data(),
                                      static_cast<int>(indices.size()), &opt, &syn),
                  "AtomGraphSynthesis::upload");
    precision = prec;
  }

  bool isUploaded() const { return syn != nullptr; }
  PrecisionModel getPrecisionModel() const { return precision; }

  /* STORMM's AtomGraphSynthesis::loadNonbondedWorkUnits (atomgraph_synthesis.h:429-431): the
   * nonbonded work units exactly as STORMM builds them, for callers that keep STORMM's launch
   * data (the kernels here use their own).  The mask synthesis argument stands for the
   * exclusions of this synthesis' topologies. */
  void loadNonbondedWorkUnits(const class StaticExclusionMaskSynthesis &,
                              InitializationTask init_request = InitializationTask::NONE,
                              int random_cache_depth = 0, const GpuDetails & = GpuDetails()) {
    std::vector<sb_topology> tops;
    for (AtomGraph* ag : topologies) {
      tops.push_back(ag->abi());
    }
    long long na = 0, ni = 0;
    const int task = static_cast<int>(init_request);
    detail::check(sb_nonbonded_work_units(tops.data(), static_cast<int>(tops.size()),
                                          indices.data(), static_cast<int>(indices.size()), task,
                                          random_cache_depth, nullptr, &na, nullptr, &ni),
                  "AtomGraphSynthesis::loadNonbondedWorkUnits");
    nbwu_abstracts.assign(static_cast<size_t>(na), 0);
    nbwu_instructions.assign(static_cast<size_t>(ni), 0u);
    detail::check(sb_nonbonded_work_units(tops.data(), static_cast<int>(tops.size()),
                                          indices.data(), static_cast<int>(indices.size()), task,
                                          random_cache_depth, nbwu_abstracts.data(), &na,
                                          nbwu_instructions.data(), &ni),
                  "AtomGraphSynthesis::loadNonbondedWorkUnits");
  }
  int getNonbondedWorkUnitCount() const { return static_cast<int>(nbwu_abstracts.size() / 64); }
  /* 64 ints per work unit, STORMM's TILE_GROUPS abstract layout */
  const std::vector<int> &getNonbondedWorkUnitAbstracts() const { return nbwu_abstracts; }
  /* (x, y) words of each tile instruction, each unit's list padded to a multiple of 32 */
  const std::vector<uint32_t> &getNonbondedWorkUnitInstructions() const {
    return nbwu_instructions;
  }

  /* The device synthesis (throws before upload) */
  sb_synthesis* handle() const {
    if (syn == nullptr) {
      throw std::runtime_error("AtomGraphSynthesis: upload() has not been called");
    }
    return syn;
  }

private:
  friend class PhaseSpaceSynthesis;
  std::vector<AtomGraph*> topologies;
  std::vector<int> indices;
  sb_options opt{};
  std::vector<double> neck_sep, neck_val;
  ImplicitSolventModel model = ImplicitSolventModel::NONE;
  PrecisionModel precision = PrecisionModel::SINGLE;
  sb_synthesis* syn = nullptr;
  mutable const void* bound_coordinates = nullptr;
  std::vector<int> nbwu_abstracts;
  std::vector<uint32_t> nbwu_instructions;

  static std::vector<int> identity(size_t n) {
    std::vector<int> v(n);
    for (size_t i = 0; i < n; i++) {
      v[i] = static_cast<int>(i);
    }
    return v;
  }

  void requireNotUploaded(const char* what) const {
    if (syn != nullptr) {
      throw std::runtime_error(std::string("AtomGraphSynthesis::") + what +
                               ": the synthesis is already on the device");
    }
  }

  void applyModel(ImplicitSolventModel igb_in, AtomicRadiusSet radii_set, double dielectric_in,
                  double saltcon_in) {
    requireNotUploaded("setImplicitSolventModel");
    for (AtomGraph* ag : topologies) {
      ag->setImplicitSolventModel(igb_in, dielectric_in, saltcon_in, radii_set);
    }
    model = igb_in;
    opt.igb = detail::igbNumber(igb_in);
    opt.dielectric = dielectric_in;
    opt.saltcon = saltcon_in;
  }
};

/* STORMM's PhaseSpaceSynthesis: coordinates and forces of every system, host side here; the
 * device side lives in the AtomGraphSynthesis it is launched with */
class PhaseSpaceSynthesis {
public:
  PhaseSpaceSynthesis(const std::vector<PhaseSpace> &ps_list,
                      const std::vector<AtomGraph*> &ag_list)
      : PhaseSpaceSynthesis(ps_list, ag_list, identity(ps_list.size())) {}

  PhaseSpaceSynthesis(const std::vector<PhaseSpace> &ps_list,
                      const std::vector<AtomGraph*> &ag_list, const std::vector<int> &index_key) {
    if (ps_list.size() != ag_list.size()) {
      throw std::runtime_error("PhaseSpaceSynthesis: one topology per coordinate set is "
                               "required");
    }
    offsets.push_back(0);
    for (int k : index_key) {
      if (k < 0 || k >= static_cast<int>(ps_list.size())) {
        throw std::runtime_error("PhaseSpaceSynthesis: index key out of range");
      }
      const PhaseSpace &ps = ps_list[static_cast<size_t>(k)];
      if (ag_list[static_cast<size_t>(k)] == nullptr ||
          ag_list[static_cast<size_t>(k)]->getAtomCount() != ps.getAtomCount()) {
        throw std::runtime_error("PhaseSpaceSynthesis: coordinates and topology of system " +
                                 std::to_string(counts.size()) + " differ in atom count");
      }
      counts.push_back(ps.getAtomCount());
      offsets.push_back(offsets.back() + ps.getAtomCount());
      xyz.insert(xyz.end(), ps.xyz.begin(), ps.xyz.end());
    }
    frc.assign(xyz.size(), 0.0);
    upload_pending = true;
  }

  int getSystemCount() const { return static_cast<int>(counts.size()); }
  int getAtomCount(int system) const { return counts.at(static_cast<size_t>(system)); }

  /* Host coordinates to the device (now if bound, else when first launched) */
  void upload() {
    upload_pending = true;
    flush(nullptr);
  }

  /* Device coordinates and forces to the host */
  void download() {
    sb_synthesis* h = boundHandle("download");
    detail::check(sb_get_coordinates(h, xyz.data(), stream), "PhaseSpaceSynthesis::download");
    detail::check(sb_get_forces(h, frc.data(), stream), "PhaseSpaceSynthesis::download");
  }

  /* Zero the force accumulators (now if bound, else when first launched) */
  void initializeForces() {
    init_pending = true;
    flush(nullptr);
  }

  std::vector<double> getInterlacedCoordinates(
      int system_index, TrajectoryKind kind = TrajectoryKind::POSITIONS) const {
    const size_t s = static_cast<size_t>(system_index);
    const size_t a = 3 * static_cast<size_t>(offsets.at(s));
    const size_t b = 3 * static_cast<size_t>(offsets.at(s + 1));
    if (kind == TrajectoryKind::VELOCITIES) {
      return std::vector<double>(b - a, 0.0);
    }
    const std::vector<double> &src = (kind == TrajectoryKind::FORCES) ? frc : xyz;
    return std::vector<double>(src.begin() + static_cast<long>(a),
                               src.begin() + static_cast<long>(b));
  }

  PhaseSpace exportSystem(int index) const {
    PhaseSpace ps(getAtomCount(index), getInterlacedCoordinates(index));
    ps.frc = getInterlacedCoordinates(index, TrajectoryKind::FORCES);
    return ps;
  }

  void importSystem(const PhaseSpace &ps, int index) {
    if (ps.getAtomCount() != getAtomCount(index)) {
      throw std::runtime_error("PhaseSpaceSynthesis::importSystem: atom count differs");
    }
    std::copy(ps.xyz.begin(), ps.xyz.end(),
              xyz.begin() + 3 * static_cast<long>(offsets[static_cast<size_t>(index)]));
    upload_pending = true;
  }

  /* Attach to a synthesis and carry out pending uploads / initializations on the stream */
  void bind(const AtomGraphSynthesis &ag, void* launch_stream) {
    sb_synthesis* h = ag.handle();
    if (ag.getSystemCount() != getSystemCount()) {
      throw std::runtime_error("PhaseSpaceSynthesis: system count differs from the topology "
                               "synthesis");
    }
    for (int s = 0; s < getSystemCount(); s++) {
      if (ag.getAtomCount(s) != counts[static_cast<size_t>(s)]) {
        throw std::runtime_error("PhaseSpaceSynthesis: atom count of system " +
                                 std::to_string(s) + " differs from the topology synthesis");
      }
    }
    if (ag.bound_coordinates != this) {
      upload_pending = true;
      ag.bound_coordinates = this;
    }
    syn = h;
    stream = launch_stream;
    flush(launch_stream);
  }

private:
  std::vector<int> counts, offsets;
  std::vector<double> xyz, frc;
  bool upload_pending = false, init_pending = false;
  sb_synthesis* syn = nullptr;
  void* stream = nullptr;

  static std::vector<int> identity(size_t n) {
    std::vector<int> v(n);
    for (size_t i = 0; i < n; i++) {
      v[i] = static_cast<int>(i);
    }
    return v;
  }

  sb_synthesis* boundHandle(const char* what) const {
    if (syn == nullptr) {
      throw std::runtime_error(std::string("PhaseSpaceSynthesis::") + what +
                               ": not yet launched with a synthesis");
    }
    return syn;
  }

  void flush(void* s) {
    if (syn == nullptr) {
      return;
    }
    if (upload_pending) {
      detail::check(sb_set_coordinates(syn, xyz.data(), s), "PhaseSpaceSynthesis::upload");
      upload_pending = false;
    }
    if (init_pending) {
      detail::check(sb_initialize(syn, SB_INIT_FORCES, s), "PhaseSpaceSynthesis::initializeForces");
      init_pending = false;
    }
  }
};

/* STORMM's StaticExclusionMaskSynthesis: the exclusion masks are built into the device
 * synthesis (32 x 32 tiles); STORMM's own tables are available per topology through
 * sb_static_exclusion_mask */
class StaticExclusionMaskSynthesis {
public:
  explicit StaticExclusionMaskSynthesis(const AtomGraphSynthesis &poly_ag) : ag(&poly_ag) {}
  StaticExclusionMaskSynthesis(const std::vector<AtomGraph*> &, const std::vector<int> &) {}
  const AtomGraphSynthesis* getTopologySynthesis() const { return ag; }
private:
  const AtomGraphSynthesis* ag = nullptr;
};

/* STORMM's CoreKlManager (Structure/core_kernel_manager.h:83): launch shapes are tuned inside
 * the library (sb_autotune); this carries the stream the launches go to */
class CoreKlManager {
public:
  CoreKlManager(const GpuDetails &gpu = GpuDetails(), void* stream_in = nullptr)
      : device(gpu.getDeviceIndex()), stream(stream_in) {}
  CoreKlManager(const GpuDetails &gpu, const AtomGraphSynthesis &, void* stream_in = nullptr)
      : CoreKlManager(gpu, stream_in) {}
  void setStream(void* stream_in) { stream = stream_in; }
  void* getStream() const { return stream; }
  int getDeviceIndex() const { return device; }
private:
  int device;
  void* stream;
};

/* ------------------------------------------------------------------------------------------ */
/* Energies and GB workspace                                                                   */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's ScoreCard (Potential/scorecard.h:101): int64 energies per system and state variable
 * with nrg_scale_bits fraction bits; the device accumulators are the synthesis' */
class ScoreCard {
public:
  explicit ScoreCard(int system_count_in, int capacity_in = 16,
                     int nrg_scale_bits_in = default_energy_scale_bits)
      : nsys(system_count_in), capacity(capacity_in), bits(nrg_scale_bits_in),
        fixed(static_cast<size_t>(system_count_in) * SB_NRG_STRIDE, 0),
        history(static_cast<size_t>(system_count_in)) {
    if (nsys <= 0) {
      throw std::runtime_error("ScoreCard: at least one system is required");
    }
  }

  int getSystemCount() const { return nsys; }
  int getEnergyScaleBits() const { return bits; }
  int getCapacity() const { return capacity; }
  int getSampleSize() const { return history.empty() ? 0 : static_cast<int>(history[0].size()); }

  /* Zero the device accumulators (now if bound, else when first launched) and the host copy */
  void initialize() {
    std::fill(fixed.begin(), fixed.end(), 0);
    init_pending = true;
    flush(nullptr);
  }

  /* Device energies to the host */
  void download() {
    if (syn == nullptr) {
      throw std::runtime_error("ScoreCard::download: not yet launched with a synthesis");
    }
    detail::check(sb_get_energies_fixed(syn, fixed.data(), stream), "ScoreCard::download");
  }

  double reportInstantaneousStates(StateVariable aspect, int system_index) const {
    checkSystem(system_index);
    const int64_t* e = &fixed[static_cast<size_t>(system_index) * SB_NRG_STRIDE];
    const int v = static_cast<int>(aspect);
    if (aspect == StateVariable::POTENTIAL_ENERGY || aspect == StateVariable::TOTAL_ENERGY) {
      int64_t sum = 0;
      for (int k = 0; k <= static_cast<int>(StateVariable::RESTRAINT); k++) {
        sum += e[k];
      }
      return std::ldexp(static_cast<double>(sum), -bits);
    }
    if (v >= 0 && v < SB_NRG_STRIDE) {
      return std::ldexp(static_cast<double>(e[v]), -bits);
    }
    return 0.0;
  }

  std::vector<double> reportInstantaneousStates(int system_index) const {
    std::vector<double> out;
    for (int v = 0; v < static_cast<int>(StateVariable::ALL_STATES); v++) {
      out.push_back(reportInstantaneousStates(static_cast<StateVariable>(v), system_index));
    }
    return out;
  }

  std::vector<double> reportInstantaneousStates(StateVariable aspect) const {
    std::vector<double> out;
    for (int s = 0; s < nsys; s++) {
      out.push_back(reportInstantaneousStates(aspect, s));
    }
    return out;
  }

  double reportPotentialEnergy(int system_index = 0) const {
    return reportInstantaneousStates(StateVariable::POTENTIAL_ENERGY, system_index);
  }
  std::vector<double> reportPotentialEnergies() const {
    return reportInstantaneousStates(StateVariable::POTENTIAL_ENERGY);
  }
  double reportTotalEnergy(int system_index = 0) const {
    return reportPotentialEnergy(system_index);
  }
  std::vector<double> reportTotalEnergies() const { return reportPotentialEnergies(); }

  /* Total energy at each recorded sample (launchMinimization records one every
   * getDiagnosticPrintFrequency() cycles and the final energy) */
  std::vector<double> reportHistory(int system_index) const {
    checkSystem(system_index);
    return history[static_cast<size_t>(system_index)];
  }
  std::vector<double> reportHistory(StateVariable aspect, int system_index) const {
    if (aspect != StateVariable::POTENTIAL_ENERGY && aspect != StateVariable::TOTAL_ENERGY) {
      throw std::runtime_error("ScoreCard::reportHistory: only the total energy is recorded");
    }
    return reportHistory(system_index);
  }

  const std::vector<int64_t> &fixedPointEnergies() const { return fixed; }

  void bind(const AtomGraphSynthesis &ag, void* launch_stream) {
    if (ag.getSystemCount() != nsys) {
      throw std::runtime_error("ScoreCard: system count differs from the topology synthesis");
    }
    if (ag.getEnergyScaleBits() != bits) {
      throw std::runtime_error("ScoreCard: energy scale bits (" + std::to_string(bits) +
                               ") differ from the synthesis' (" +
                               std::to_string(ag.getEnergyScaleBits()) + ")");
    }
    syn = ag.handle();
    stream = launch_stream;
    flush(launch_stream);
  }

  void setHistory(std::vector<std::vector<double>> samples) { history = std::move(samples); }

private:
  int nsys, capacity, bits;
  std::vector<int64_t> fixed;
  std::vector<std::vector<double>> history;
  bool init_pending = false;
  sb_synthesis* syn = nullptr;
  void* stream = nullptr;

  void checkSystem(int s) const {
    if (s < 0 || s >= nsys) {
      throw std::runtime_error("ScoreCard: system index " + std::to_string(s) +
                               " out of range");
    }
  }

  void flush(void* s) {
    if (syn != nullptr && init_pending) {
      detail::check(sb_initialize(syn, SB_INIT_ENERGIES, s), "ScoreCard::initialize");
      init_pending = false;
    }
  }
};

/* STORMM's ImplicitSolventWorkspace (Potential/implicit_solvent_workspace.h:17-120): psi and
 * sum of dE/dR accumulators, the synthesis' own */
class ImplicitSolventWorkspace {
public:
  explicit ImplicitSolventWorkspace(const AtomGraphSynthesis &poly_ag,
                                    PrecisionModel prec = PrecisionModel::SINGLE)
      : ag(&poly_ag), precision(prec) {}

  /* Zero the accumulators (now if the synthesis is on the device, else at the first launch) */
  void initialize() {
    init_pending = true;
    flush(nullptr);
  }

  /* psi (A^-1), effective radii (A) and sum of dE/dR per atom, all systems back to back */
  void download() {
    size_t n = 0;
    for (int s = 0; s < ag->getSystemCount(); s++) {
      n += static_cast<size_t>(ag->getAtomCount(s));
    }
    psi.assign(n, 0.0);
    radii.assign(n, 0.0);
    sumdeijda.assign(n, 0.0);
    detail::check(sb_get_gb_workspace(ag->handle(), psi.data(), radii.data(), sumdeijda.data(),
                                      stream),
                  "ImplicitSolventWorkspace::download");
  }
  const std::vector<double> &getPsi() const { return psi; }
  const std::vector<double> &getEffectiveRadii() const { return radii; }
  const std::vector<double> &getSumDeijda() const { return sumdeijda; }
  PrecisionModel getPrecisionModel() const { return precision; }

  void bind(const AtomGraphSynthesis &poly_ag, void* launch_stream) {
    if (&poly_ag != ag) {
      throw std::runtime_error("ImplicitSolventWorkspace: launched with another synthesis than "
                               "the one it was made for");
    }
    stream = launch_stream;
    flush(launch_stream);
  }

private:
  const AtomGraphSynthesis* ag;
  PrecisionModel precision;
  std::vector<double> psi, radii, sumdeijda;
  bool init_pending = false;
  void* stream = nullptr;

  void flush(void* s) {
    if (init_pending && ag->isUploaded()) {
      detail::check(sb_initialize(ag->handle(), SB_INIT_GB_WORKSPACE, s),
                    "ImplicitSolventWorkspace::initialize");
      init_pending = false;
    }
  }
};

/* ------------------------------------------------------------------------------------------ */
/* Minimization controls                                                                       */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's MinimizeControls (Namelists/nml_minimize.h:21-175) with its defaults */
class MinimizeControls {
public:
  MinimizeControls() = default;
  int getTotalCycles() const { return maxcyc; }
  int getSteepestDescentCycles() const { return ncyc; }
  int getClashDampingCycles() const { return cdcyc; }
  int getDiagnosticPrintFrequency() const { return ntpr; }
  double getInitialStep() const { return dx0; }
  double getConvergenceTarget() const { return drms; }
  double getAbsoluteClashDistance() const { return clash_r0; }
  double getVdwClashRatio() const { return clash_ratio; }
  void setTotalCycles(int cycles_in) { maxcyc = positive(cycles_in, "total cycles"); }
  void setSteepestDescentCycles(int cycles_in) { ncyc = nonNegative(cycles_in, "SD cycles"); }
  void setClashDampingCycles(int cycles_in) { cdcyc = nonNegative(cycles_in, "clash cycles"); }
  void setDiagnosticPrintFrequency(int frequency_in) { ntpr = frequency_in; }
  void setInitialStep(double step_size_in) {
    if (!(step_size_in > 0.0)) {
      throw std::runtime_error("MinimizeControls: the initial step must be positive");
    }
    dx0 = step_size_in;
  }
  void setConvergenceTarget(double target_in) { drms = target_in; }
  void setAbsoluteClashDistance(double d) { clash_r0 = d; }
  void setVdwClashRatio(double r) { clash_ratio = r; }

private:
  int maxcyc = 200, ncyc = 50, cdcyc = 25, ntpr = 0;
  double dx0 = 0.01, drms = 0.0001, clash_r0 = 0.2, clash_ratio = 0.5;

  static int positive(int v, const char* what) {
    if (v <= 0) {
      throw std::runtime_error(std::string("MinimizeControls: ") + what + " must be positive");
    }
    return v;
  }
  static int nonNegative(int v, const char* what) {
    if (v < 0) {
      throw std::runtime_error(std::string("MinimizeControls: ") + what +
                               " must not be negative");
    }
    return v;
  }
};

inline MolecularMechanicsControls::MolecularMechanicsControls(const MinimizeControls &user_input)
    : total_cycles(user_input.getTotalCycles()),
      sd_cycles(user_input.getSteepestDescentCycles()),
      initial_step(user_input.getInitialStep()) {}

/* ------------------------------------------------------------------------------------------ */
/* Launchers                                                                                   */
/* ------------------------------------------------------------------------------------------ */
namespace detail {

inline sb_synthesis* prepare(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                             PhaseSpaceSynthesis* poly_ps, ScoreCard* sc,
                             ImplicitSolventWorkspace* ism_space, void* stream,
                             const char* who) {
  sb_synthesis* h = poly_ag.handle();
  if (prec != poly_ag.getPrecisionModel()) {
    throw std::runtime_error(std::string(who) + ": the synthesis was uploaded for the other "
                             "precision model");
  }
  if (poly_ps == nullptr) {
    throw std::runtime_error(std::string(who) + ": a PhaseSpaceSynthesis is required");
  }
  poly_ps->bind(poly_ag, stream);
  if (sc != nullptr) {
    sc->bind(poly_ag, stream);
  }
  if (ism_space != nullptr) {
    ism_space->bind(poly_ag, stream);
  }
  return h;
}

}  // namespace detail

/* launchNonbonded (Potential/hpc_nonbonded_potential.h:142-157): Coulomb, Lennard-Jones and the
 * GB passes of every system, forces into the PhaseSpaceSynthesis and energies into the
 * ScoreCard (accumulated: initialize them first) */
inline void launchNonbonded(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                            const StaticExclusionMaskSynthesis &, MolecularMechanicsControls *,
                            PhaseSpaceSynthesis *poly_ps, Thermostat *, ScoreCard *sc,
                            CacheResource *, ImplicitSolventWorkspace *ism_space,
                            EvaluateForce eval_force, EvaluateEnergy eval_energy,
                            AccumulationMethod, const CoreKlManager &launcher,
                            double clash_minimum_distance = 0.0, double clash_ratio = 0.0) {
  void* stream = launcher.getStream();
  sb_synthesis* h = detail::prepare(prec, poly_ag, poly_ps, sc, ism_space, stream,
                                    "launchNonbonded");
  const int terms = SB_TERM_NONBONDED |
                    (poly_ag.getImplicitSolventModel() != ImplicitSolventModel::NONE ?
                     SB_TERM_GB : 0);
  detail::check(sb_evaluate_clash(h, terms, eval_force == EvaluateForce::YES,
                                  eval_energy == EvaluateEnergy::YES, clash_minimum_distance,
                                  clash_ratio, stream),
                "launchNonbonded");
}

inline void launchNonbonded(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                            const StaticExclusionMaskSynthesis &poly_se,
                            MolecularMechanicsControls *mmctrl, PhaseSpaceSynthesis *poly_ps,
                            Thermostat *heat_bath, ScoreCard *sc, CacheResource *tb_space,
                            ImplicitSolventWorkspace *ism_space, EvaluateForce eval_force,
                            EvaluateEnergy eval_energy, const CoreKlManager &launcher,
                            double clash_minimum_distance = 0.0, double clash_ratio = 0.0) {
  launchNonbonded(prec, poly_ag, poly_se, mmctrl, poly_ps, heat_bath, sc, tb_space, ism_space,
                  eval_force, eval_energy, AccumulationMethod::SPLIT, launcher,
                  clash_minimum_distance, clash_ratio);
}

/* launchValence (Potential/hpc_valence_potential.h:305-317): bonds, angles, dihedrals and the
 * attenuated 1-4 pairs of every system.  VwuGoal::MOVE_PARTICLES (dynamics) is outside this
 * path. */
inline void launchValence(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                          MolecularMechanicsControls *, PhaseSpaceSynthesis *poly_ps,
                          Thermostat *, ScoreCard *sc, CacheResource *, EvaluateForce eval_force,
                          EvaluateEnergy eval_energy, VwuGoal purpose, AccumulationMethod,
                          const CoreKlManager &launcher, double clash_distance = 0.0,
                          double clash_ratio = 0.0) {
  if (purpose != VwuGoal::ACCUMULATE) {
    throw std::runtime_error("launchValence: only VwuGoal::ACCUMULATE is supported (no "
                             "particle moves in this path)");
  }
  void* stream = launcher.getStream();
  sb_synthesis* h = detail::prepare(prec, poly_ag, poly_ps, sc, nullptr, stream,
                                    "launchValence");
  detail::check(sb_evaluate_clash(h, SB_TERM_VALENCE, eval_force == EvaluateForce::YES,
                                  eval_energy == EvaluateEnergy::YES, clash_distance,
                                  clash_ratio, stream),
                "launchValence");
}

inline void launchValence(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                          MolecularMechanicsControls *mmctrl, PhaseSpaceSynthesis *poly_ps,
                          Thermostat *heat_bath, ScoreCard *sc, CacheResource *tb_space,
                          EvaluateForce eval_force, EvaluateEnergy eval_energy, VwuGoal purpose,
                          const CoreKlManager &launcher, double clash_distance = 0.0,
                          double clash_ratio = 0.0) {
  launchValence(prec, poly_ag, mmctrl, poly_ps, heat_bath, sc, tb_space, eval_force,
                eval_energy, purpose, AccumulationMethod::SPLIT, launcher, clash_distance,
                clash_ratio);
}

/* launchConjugateGradient (Math/hpc_reduction.h:55-63): after a force + energy evaluation at the
 * line start, one conjugate-gradient step of every system (sb_conjugate_gradient: gg, dgg, the
 * steepest-descent / conjugate-gradient switch after mmctrl's steepest-descent cycles, the new
 * search direction).  The first call with a given MolecularMechanicsControls begins the
 * synthesis' minimizer state from it (move length, no previous direction, zero cycles). */
inline void launchConjugateGradient(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                                    PhaseSpaceSynthesis *poly_ps, ReductionBridge *,
                                    MolecularMechanicsControls *mmctrl,
                                    const CoreKlManager &launcher) {
  void* stream = launcher.getStream();
  sb_synthesis* h = detail::prepare(prec, poly_ag, poly_ps, nullptr, nullptr, stream,
                                    "launchConjugateGradient");
  if (mmctrl == nullptr) {
    throw std::runtime_error("launchConjugateGradient: MolecularMechanicsControls required");
  }
  if (mmctrl->begunFor() != h) {
    sb_minimize_controls c;
    sb_default_minimize_controls(&c);
    c.total_cycles = mmctrl->getTotalCycles();
    c.sd_cycles = mmctrl->getSteepestDescentCycles();
    c.initial_step = mmctrl->getInitialStep();
    c.clash_cycles = 0;
    c.convergence_rms = 0.0;
    c.kernel = SB_MIN_GRAPH;
    detail::check(sb_minimize_begin(h, &c, stream), "launchConjugateGradient");
    mmctrl->markBegun(h);
  }
  detail::check(sb_conjugate_gradient(h, stream), "launchConjugateGradient");
}

/* launchLineAdvance (MolecularMechanics/hpc_minimization.h:63-70): move 0-3 of the line search
 * after an energy evaluation at the current coordinates (sb_line_advance); the energies are read
 * on the device, so the ScoreCard is only bound */
inline void launchLineAdvance(PrecisionModel prec, PhaseSpaceSynthesis *poly_ps,
                              const AtomGraphSynthesis &poly_ag, ScoreCard *sc,
                              LineMinimization *line_record, int move_number,
                              const CoreKlManager &launcher) {
  void* stream = launcher.getStream();
  sb_synthesis* h = detail::prepare(prec, poly_ag, poly_ps, sc, nullptr, stream,
                                    "launchLineAdvance");
  if (line_record != nullptr && line_record->getSystemCount() != poly_ag.getSystemCount()) {
    throw std::runtime_error("launchLineAdvance: the LineMinimization record is for another "
                             "system count");
  }
  detail::check(sb_line_advance(h, move_number, stream), "launchLineAdvance");
}

namespace detail {

/* The minimization itself, shared by the launchMinimization overloads */
inline void minimize(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                     PhaseSpaceSynthesis *poly_ps, const MinimizeControls &mincon, ScoreCard *sc,
                     void* stream) {
  sb_synthesis* h = prepare(prec, poly_ag, poly_ps, sc, nullptr, stream, "launchMinimization");
  sb_minimize_controls c;
  sb_default_minimize_controls(&c);
  c.total_cycles = mincon.getTotalCycles();
  c.sd_cycles = mincon.getSteepestDescentCycles();
  c.clash_cycles = mincon.getClashDampingCycles();
  c.clash_distance = mincon.getAbsoluteClashDistance();
  c.clash_ratio = mincon.getVdwClashRatio();
  c.initial_step = mincon.getInitialStep();
  c.convergence_rms = 0.0;                 // STORMM's GPU minimizer runs every cycle
  const int ntpr = mincon.getDiagnosticPrintFrequency();
  c.record_history = (ntpr > 0) ? 1 : 0;
  check(sb_minimize(h, &c, stream), "launchMinimization");
  if (sc == nullptr) {
    return;
  }
  sc->download();
  const int nsys = poly_ag.getSystemCount();
  std::vector<std::vector<double>> samples(static_cast<size_t>(nsys));
  if (ntpr > 0) {
    const int stride = c.total_cycles + 1;
    std::vector<double> hist(static_cast<size_t>(nsys) * stride);
    check(sb_get_minimize_history(h, hist.data(), stream), "launchMinimization");
    for (int s = 0; s < nsys; s++) {
      for (int cyc = 0; cyc < c.total_cycles; cyc += ntpr) {
        samples[static_cast<size_t>(s)].push_back(hist[static_cast<size_t>(s) * stride + cyc]);
      }
      samples[static_cast<size_t>(s)].push_back(
          hist[static_cast<size_t>(s) * stride + c.total_cycles]);
    }
  }
  else {
    for (int s = 0; s < nsys; s++) {
      samples[static_cast<size_t>(s)].push_back(sc->reportTotalEnergy(s));
    }
  }
  sc->setHistory(std::move(samples));
}

}  // namespace detail

/* launchMinimization (MolecularMechanics/hpc_minimization.h:122-152): steepest descent, then
 * conjugate gradient with a four-point line search, clash-damped for the first
 * getClashDampingCycles() cycles; coordinates move in place on the device (download the
 * PhaseSpaceSynthesis to read them) and the ScoreCard receives the final energies and the
 * total energy every getDiagnosticPrintFrequency() cycles.  With PrecisionModel::DOUBLE the
 * synthesis must have been uploaded for FP64. */
inline void launchMinimization(PrecisionModel prec, const AtomGraphSynthesis &poly_ag,
                               const StaticExclusionMaskSynthesis &, PhaseSpaceSynthesis *poly_ps,
                               const MinimizeControls &mincon, MolecularMechanicsControls *,
                               MolecularMechanicsControls *, MolecularMechanicsControls *,
                               MolecularMechanicsControls *, ScoreCard *sc, CacheResource *,
                               CacheResource *, CacheResource *, CacheResource *, CacheResource *,
                               CacheResource *, ImplicitSolventWorkspace *, ReductionBridge *,
                               LineMinimization *, AccumulationMethod, const GpuDetails &,
                               const CoreKlManager &launcher, StopWatch * = nullptr,
                               const std::string & = std::string("")) {
  detail::minimize(prec, poly_ag, poly_ps, mincon, sc, launcher.getStream());
}

inline ScoreCard launchMinimization(const AtomGraphSynthesis &poly_ag,
                                    const StaticExclusionMaskSynthesis &,
                                    PhaseSpaceSynthesis *poly_ps, const MinimizeControls &mincon,
                                    const GpuDetails &, PrecisionModel prec = PrecisionModel::SINGLE,
                                    int energy_accumulation_bits = default_energy_scale_bits,
                                    StopWatch * = nullptr, const std::string & = std::string("")) {
  const int ntpr = mincon.getDiagnosticPrintFrequency();
  const int frames = (ntpr > 0) ? (mincon.getTotalCycles() + ntpr - 1) / ntpr + 1 : 1;
  ScoreCard result(poly_ag.getSystemCount(), frames, energy_accumulation_bits);
  detail::minimize(prec, poly_ag, poly_ps, mincon, &result, nullptr);
  return result;
}

inline ScoreCard launchMinimization(const AtomGraphSynthesis &poly_ag,
                                    PhaseSpaceSynthesis *poly_ps, const MinimizeControls &mincon,
                                    const GpuDetails &gpu,
                                    PrecisionModel prec = PrecisionModel::SINGLE,
                                    int energy_accumulation_bits = default_energy_scale_bits,
                                    StopWatch *timer = nullptr,
                                    const std::string &task_name = std::string("")) {
  return launchMinimization(poly_ag, StaticExclusionMaskSynthesis(poly_ag), poly_ps, mincon, gpu,
                            prec, energy_accumulation_bits, timer, task_name);
}

}  // namespace stormm_b200

#endif
