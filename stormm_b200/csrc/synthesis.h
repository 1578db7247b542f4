// Host-side synthesis of many molecules for the batched implicit-solvent path.
//
// One object holds what STORMM spreads over AtomGraphSynthesis (parameters, valence terms,
// Lennard-Jones tables: Synthesis/atomgraph_synthesis.h:55), StaticExclusionMaskSynthesis
// (exclusions, Synthesis/static_mask_synthesis.h:54), PhaseSpaceSynthesis (fixed-point
// coordinates and forces, Synthesis/phasespace_synthesis.h:325), ImplicitSolventWorkspace
// (Synthesis/implicit_solvent_workspace.h:65) and ScoreCard (Potential/scorecard.h:101) for this
// path, as device arrays in the layout described in device_kits.h.
#ifndef STORMM_B200_SYNTHESIS_H
#define STORMM_B200_SYNTHESIS_H

#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "stormm_b200.h"
#include "device_kits.h"

namespace sb {

class Error : public std::runtime_error {
public:
  Error(int code_in, const std::string &msg) : std::runtime_error(msg), code(code_in) {}
  int code;
};

void cudaCheck(cudaError_t err, const char* what);
void setLastError(const std::string &msg);
const char* lastError();

// Stream for stream-ordered allocation by the calling thread; null (the default) means plain
// cudaMalloc / cudaFree.  The request server sets it while it builds or retires a batch, so that
// allocating and freeing device memory does not wait for the other batches' kernels.
cudaStream_t &allocationStream();

class AllocationStreamGuard {
public:
  explicit AllocationStreamGuard(cudaStream_t s) : prev_(allocationStream()) {
    allocationStream() = s;
  }
  ~AllocationStreamGuard() { allocationStream() = prev_; }
private:
  cudaStream_t prev_;
};

// Device array owned by the synthesis
template <typename T> struct DeviceArray {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;      // stream of a stream-ordered allocation
  bool owned = true;             // false: a view into another array's memory (UploadArena)
  DeviceArray() = default;
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray& operator=(const DeviceArray &) = delete;
  ~DeviceArray() { release(); }
  void release() {
    if (p != nullptr && owned) {
      if (s != nullptr) {
        cudaFreeAsync(p, s);
      }
      else {
        cudaFree(p);
      }
    }
    p = nullptr;
    owned = true;
  }
  void view(T* ptr, size_t count) {
    release();
    p = ptr;
    n = count;
    owned = false;
  }
  void allocate(size_t count) {
    release();
    n = count;
    s = allocationStream();
    const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    if (s != nullptr) {
      cudaCheck(cudaMallocAsync(reinterpret_cast<void**>(&p), bytes, s), "cudaMallocAsync");
      // usable by the synchronous copies that follow
      cudaCheck(cudaStreamSynchronize(s), "cudaMallocAsync");
    }
    else {
      cudaCheck(cudaMalloc(reinterpret_cast<void**>(&p), bytes), "cudaMalloc");
    }
  }
  void zeros(size_t count) {
    allocate(count);
    // ordered on the allocation stream and waited for, as the next user may be another stream
    cudaCheck(cudaMemsetAsync(p, 0, sizeof(T) * (count > 0 ? count : 1), s), "cudaMemsetAsync");
    cudaCheck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  void upload(const std::vector<T> &v) {
    allocate(v.size());
    if (!v.empty()) {
      cudaCheck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice),
                "cudaMemcpy");
    }
  }
};

// Many device arrays built at once: one allocation holds them all (256-byte aligned), the
// arrays with host contents arrive in one copy and the zeroed ones are cleared by one memset,
// instead of an allocation, a synchronization and a copy or memset per array.  The arrays
// become views into `block`, which owns the memory.
class UploadArena {
public:
  template <typename T> void put(DeviceArray<T>* a, const std::vector<T> &v) {
    add(&up_, v.empty() ? nullptr : v.data(), sizeof(T) * v.size(), sizeof(T),
        [a, n = v.size()](unsigned char* at) { a->view(reinterpret_cast<T*>(at), n); });
  }
  template <typename T> void zero(DeviceArray<T>* a, size_t count) {
    add(&zero_, nullptr, sizeof(T) * count, sizeof(T),
        [a, count](unsigned char* at) { a->view(reinterpret_cast<T*>(at), count); });
  }
  void commit(DeviceArray<unsigned char>* block);
private:
  struct Item {
    const void* src;
    size_t bytes;
    std::function<void(unsigned char*)> bind;
  };
  static void add(std::vector<Item>* list, const void* src, size_t bytes, size_t unit,
                  std::function<void(unsigned char*)> bind) {
    // an empty array still gets one element, as DeviceArray::allocate gives it
    list->push_back({src, bytes > 0 ? bytes : unit, std::move(bind)});
  }
  std::vector<Item> up_, zero_;
};

// Host checks of a topology before anything is built from it (the constructor of Synthesis and
// the request server's submit share them): sizes, required arrays, index ranges of
// Lennard-Jones types, exclusion partners and valence atoms, and the GB and neck parameters the
// options need.  Throws Error naming topology `which` (or "the topology" when it is negative).
void validateTopology(const sb_topology &tp, const sb_options &opt, int which);

// Host checks of minimization controls (minimizeBegin and the request server's constructor)
void validateMinimizeControls(const sb_minimize_controls &ctl);

// A system's line-minimization state at a cycle boundary (FP32 path), on the host
struct MinimizerState {
  int natom = 0;
  std::vector<long long> crd[3], prv[3];
  std::vector<int> crd_ovrf[3];
  std::vector<float> cg[3];
  double l_move = 0.0;
  double rms_force = 0.0;
  int cycle = 0;
  int done = 0;
};

// Packing of molecules into work units and the launch parameters of each size class
struct UnitPlan {
  int max_slots_cap = 0;
  int max_tiles_cap = 0;
  std::vector<int4> units;       // x = first index in systems, y = count, z = slots, w = tiles
  std::vector<int> systems;
  int n_big = 0;                 // units [0, n_big) hold one molecule above the packing cap
  int big_slots = 0, big_lj = 0;
  int small_slots = 0, small_lj = 0;
  std::vector<int> meta;         // kUnitMetaFields ints per molecule row, plus a closing row
  std::vector<int4> desc;        // as units, but x = first row of the unit in meta
  DeviceArray<int4> d_units;     // desc on the device
  DeviceArray<int> d_meta;
};

// Softened-core (clash damping) setting of an evaluation: off when both distance and ratio are
// zero; with cycle set, per system as DevSynthesis::clash_cycle describes
struct Clash {
  float distance = 0.0f;
  float ratio = 0.0f;
  double distance64 = 0.0;        // the same in double, for the FP64 mode
  double ratio64 = 0.0;
  int cycles = 0;
  const int* cycle = nullptr;
  bool on() const { return distance > 0.0f || ratio > 0.0f; }
  void apply(DevSynthesis* d) const {
    d->clash_distance = distance;
    d->clash_ratio = ratio;
    d->clash_cycles = cycles;
    d->clash_cycle = cycle;
  }
};

class Synthesis {
public:
  Synthesis(const sb_topology* tops, int ntop, const int* topology_index, int nsys,
            const sb_options &options);

  void evaluate(int terms, bool force, bool energy, cudaStream_t stream,
                const Clash &clash = Clash());
  void evaluateRange(int first, int count, int terms, bool force, bool energy,
                     cudaStream_t stream, const Clash &clash = Clash());
  void initialize(int what, cudaStream_t stream);
  void setCoordinates(const double* xyz, cudaStream_t stream);
  void getCoordinates(double* xyz, cudaStream_t stream);
  void getForces(double* xyz, cudaStream_t stream);
  void getForcesFixed(long long* prim, int* ovrf, cudaStream_t stream);
  void getEnergies(double* out, cudaStream_t stream);
  // STORMM's sphere-point surface area of every system (sasa.cu); out: nsys values on the host
  void surfaceArea(const double* points, int npts, double probe, double weight, double* out,
                   cudaStream_t stream);
  std::vector<double> h_sasa_radius;   // per padded atom: half the LJ sigma of (type 0, type)
  void downloadResults(double* forces, double* energies, cudaStream_t stream);
  void setRestraints(const sb_restraint* list, int count);
  int launchThreads(int units, int terms) const;
  void getEnergiesFixed(long long* out, cudaStream_t stream);
  void getGbWorkspace(double* psi, double* radii, double* sde, cudaStream_t stream);
  int checkStatus(cudaStream_t stream);
  void minimize(const sb_minimize_controls &ctl, cudaStream_t stream);
  void minimizeBegin(const sb_minimize_controls &ctl, cudaStream_t stream);
  void minimizeAdvance(int cycles, bool final_energy, cudaStream_t stream);
  void conjugateGradient(cudaStream_t stream);
  void lineAdvance(int move, cudaStream_t stream);
  void autotune(int what, int* chosen_slots, int* chosen_tiles, double* best_ms,
                cudaStream_t stream);
  void minimizeRange(int first, int count, const sb_minimize_controls &ctl, cudaStream_t stream);
  void getMinimizeHistory(double* out, cudaStream_t stream);
  void getMinimizeProgress(int* cycles, int* converged, double* rms, cudaStream_t stream);
  // One system's minimizer state between cycles (coordinates, previous forces, conjugate
  // direction, move length, cycle count, convergence flag, RMS force), read out of this
  // synthesis or written into another one whose system has the same topology: the system then
  // continues exactly as it would have where it was
  void exportMinimizerState(int system, MinimizerState* state, cudaStream_t stream);
  void importMinimizerState(int system, const MinimizerState &state, cudaStream_t stream);

  sb_options opt;
  int nsys = 0;
  int natom_padded = 0;
  int natom_total = 0;       // atoms without padding
  int sm_count = 0;
  int max_smem_optin = 0;
  int threads = 256;
  int max_lj = 0;
  int max_unit_slots = 0;
  std::unique_ptr<UnitPlan> eval_plan;   // batched evaluation
  std::unique_ptr<UnitPlan> min_plan;    // batched minimization
  std::unique_ptr<UnitPlan> single_plan; // one unit per system, in system order
  int tiled_threshold = kMaxFusedAtoms;  // molecules above it take the tiled path
  std::vector<int> h_tiled_systems, h_tile_prefix, h_atom_prefix;
  std::vector<int> tiled_index;          // per system: index among tiled molecules, or -1
  int single_slots = 0, single_lj = 0;
  std::vector<int> topo;
  std::vector<int> atom_start;
  std::vector<int> atom_count;

  // host staging of the packed layout
  std::vector<float> h_charge, h_rho, h_srho, h_pb, h_alpha, h_beta, h_gamma;
  std::vector<double4> h_gb_radius64;
  std::vector<double> h_gb_gamma64;
  std::vector<int> h_ljidx, h_lj_start, h_lj_ntypes, h_tile_start, h_tile_mask_idx;
  std::vector<int> h_bond_start, h_angl_start, h_dihe_start;
  std::vector<float2> h_ljab, h_ljab14;
  std::vector<uint4> h_bonds, h_angles, h_dihe_a, h_dihe_b;
  std::vector<double4> h_angl64, h_dihe64;
  std::vector<double4> h_dihe14_64;
  std::vector<unsigned int> h_mask_pool;
  std::vector<long long> h_stage_ll;
  std::vector<int> h_unpadded_map;   // padded index of each unpadded atom

  // device arrays
  DeviceArray<unsigned char> d_arena;    // owns the memory of the arrays upload() builds
  DeviceArray<unsigned char> d_min_arena;  // and of the minimizer's arrays
  // CHARMM terms (charmm.cu): records in the padded layout, per-system ranges on the host
  bool has_charmm = false;
  std::vector<int4> h_ubrd, h_cimp, h_cmap, h_cmap_b;
  std::vector<double2> h_ubrd_prm, h_cimp_prm;
  std::vector<int> h_cimp_sys, h_ubrd_start, h_cimp_start, h_cmap_start;
  std::vector<int2> h_cmap_surf;
  std::vector<double> h_cmap_patch;
  DeviceArray<int4> d_ubrd, d_cimp, d_cmap, d_cmap_b;
  DeviceArray<double2> d_ubrd_prm, d_cimp_prm;
  DeviceArray<int> d_cimp_sys;
  DeviceArray<int2> d_cmap_surf;
  DeviceArray<double> d_cmap_patch;
  DevCharmm dev_charmm;
  // restraints (sb_set_restraints): records sorted by system, per-system ranges on the host
  std::vector<int> h_rst_start;
  DeviceArray<unsigned char> d_rst_arena;
  DeviceArray<int4> d_rst_atoms;
  DeviceArray<int2> d_rst_meta;
  DeviceArray<double2> d_rst_k;
  DeviceArray<double4> d_rst_r, d_rst_target;
  DeviceArray<double2> d_rst_kf;               // final stiffnesses, bounds and targets
  DeviceArray<double4> d_rst_rf, d_rst_target_f;
  DeviceArray<int2> d_rst_steps;               // initial and final steps
  int restraint_version = 0;
  DeviceArray<int> d_atom_start, d_atom_count, d_bond_start, d_angl_start, d_dihe_start;
  DeviceArray<int> d_lj_start, d_lj_ntypes, d_tile_start, d_ljidx, d_tile_mask_idx;
  DeviceArray<float> d_charge, d_rho, d_srho, d_pb, d_alpha, d_beta, d_gamma;
  DeviceArray<double4> d_gb_radius64;
  DeviceArray<double> d_gb_gamma64;
  DeviceArray<float2> d_ljab, d_ljab14;
  DeviceArray<uint4> d_bonds, d_angles, d_dihe_a, d_dihe_b;
  DeviceArray<double4> d_angl64, d_dihe64;
  DeviceArray<double4> d_dihe14_64;
  DeviceArray<unsigned int> d_mask_pool;
  DeviceArray<long long> d_xcrd, d_ycrd, d_zcrd, d_xfrc, d_yfrc, d_zfrc;
  DeviceArray<int> d_xcrd_ovrf, d_ycrd_ovrf, d_zcrd_ovrf, d_xfrc_ovrf, d_yfrc_ovrf, d_zfrc_ovrf;
  DeviceArray<unsigned long long> d_energies;
  DeviceArray<long long> d_psi, d_sumdeijda;
  DeviceArray<int> d_psi_ovrf, d_sumdeijda_ovrf, d_status;
  DeviceArray<float> d_born_radii;
  DeviceArray<float2> d_pair_deriv;
  std::vector<int> h_neck_idx;
  std::vector<float> h_neck_sep, h_neck_val;
  std::vector<double> h64_neck_sep, h64_neck_val;
  DeviceArray<int> d_neck_idx;
  DeviceArray<float> d_neck_sep, d_neck_val;
  DeviceArray<double> d64_neck_sep, d64_neck_val;
  double gb_offset = 0.09;       // baseline radius offset of the GB model
  bool neck = false;
  int fused_tiles = 0;           // tiles of all molecules on the fused path
  DeviceArray<int> d_unpadded_map;
  DeviceArray<double> d_stage_xyz, d_stage_nrg;
  DeviceArray<int> d_tiled_systems, d_tile_prefix, d_atom_prefix;
  DeviceArray<long long> d_tiled_psi, d_tiled_de;
  DeviceArray<float> d_tiled_radius, d_tiled_sde;
  DevTiled dev_tiled{};
  // FP64 mode (opt.precision == SB_PRECISION_DOUBLE): double parameters and per-atom GB state
  // (charges and 1-4 tables in double are built in both modes: FP32 valence uses them too)
  bool fp64 = false;
  std::vector<double> h64_charge, h64_rho, h64_srho, h64_pb, h64_alpha, h64_beta, h64_gamma;
  std::vector<double2> h64_ljab, h64_ljab14, h64_bond_prm, h64_angl_prm, h64_dihe_attn;
  std::vector<int2> h64_bond_atoms;
  std::vector<int4> h64_angl_atoms, h64_dihe_atoms;
  std::vector<double4> h64_dihe_prm;
  DeviceArray<double> d64_charge, d64_rho, d64_srho, d64_pb, d64_alpha, d64_beta, d64_gamma;
  DeviceArray<double2> d64_ljab, d64_ljab14, d64_bond_prm, d64_angl_prm, d64_dihe_attn;
  DeviceArray<int2> d64_bond_atoms;
  DeviceArray<int4> d64_angl_atoms, d64_dihe_atoms;
  DeviceArray<double4> d64_dihe_prm;
  DeviceArray<double> d64_radius, d64_sde;
  DevPrecise dev64{};

  // line-minimization state, allocated by the first minimization
  DeviceArray<long long> d_xprv, d_yprv, d_zprv;
  DeviceArray<float> d_xcg, d_ycg, d_zcg;
  DeviceArray<double> d_xcg64, d_ycg64, d_zcg64;   // FP64 mode: the direction in double
  double min_clash_distance = 0.0, min_clash_ratio = 0.0;   // the minimizer's, in double
  DeviceArray<double> d_lmove, d_rmsf, d_history;
  DeviceArray<int> d_mcycle, d_mdone, d_queue;
  int history_stride = 0;
  DeviceArray<double> d_line;
  DevMinimizer dev_min{};
  bool min_ready = false;
  int min_kernel = SB_MIN_GRAPH;
  int min_total_cycles = 0;
  // captured minimization cycle (graph mode) and what it was captured for
  cudaGraphExec_t cycle_graph = nullptr;
  const UnitPlan* cycle_graph_plan = nullptr;
  DevMinimizer cycle_graph_min{};   // kernel arguments the graph was captured with
  DevSynthesis cycle_graph_dev{};
  int cycle_graph_restraints = 0;
  cudaStream_t capture_stream = nullptr;
  ~Synthesis();

  DevSynthesis dev;

private:
  void buildLayout(const sb_topology* tops, int ntop);
  void buildCharmm(const sb_topology* tops, int ntop);
  void launchExtraTerms(int first, int last, bool force, bool energy, cudaStream_t stream,
                        const int* cycle = nullptr);
  // defer: leave the device copy of the plan to the caller (the constructor's UploadArena)
  std::unique_ptr<UnitPlan> makePlan(int max_slots_cap, int max_tiles_cap,
                                     bool defer = false) const;
  void finalizePlan(UnitPlan* plan, bool defer = false) const;
  bool allow_wide = true;        // 512-thread blocks for small all-term launches (autotuned)
  void launchPlan(const UnitPlan &plan, int terms, bool force, bool energy, cudaStream_t stream,
                  const Clash &clash = Clash());
  void launchMinPlan(const UnitPlan &plan, int cycles, bool final_energy, cudaStream_t stream);
  void launchTiledRange(int mol_begin, int mol_end, int terms, bool force, bool energy,
                        cudaStream_t stream, const Clash &clash = Clash());
  Clash minimizerClash() const;
  void rejectTiledMinimization(int kernel) const;
  void graphCycle(int first, int count, bool single, cudaStream_t stream);
  void graphFinalEnergy(int first, int count, bool single, cudaStream_t stream);
  void evaluateFor(int first, int count, bool single, bool force, cudaStream_t stream,
                   const Clash &clash = Clash());
  void buildUnits();
  void upload();
};

}  // namespace sb

#endif
