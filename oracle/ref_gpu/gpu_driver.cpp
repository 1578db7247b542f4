// Driver over STORMM's own CUDA library (built from the reference sources by the Makefile beside
// this file).  Test and measurement infrastructure only: it reads Amber prmtop / inpcrd files
// through STORMM's AtomGraph and PhaseSpace, assembles them into STORMM's AtomGraphSynthesis and
// PhaseSpaceSynthesis, and runs STORMM's own GPU launchers on them, so that the implementation
// under test can be compared with the reference's GPU path on the same B200 and the same inputs.
//
// Modes (each line of <list-file> is "<prmtop> <inpcrd>"; every system keeps its own topology):
//   time <list-file> <evals> [--prec single|double] [--out <out.bin>]
//       One force + energy evaluation per step, exactly the launches of the first stage of a
//       cycle of STORMM's GPU line minimizer (MolecularMechanics/hpc_minimization.cu: clear the
//       forces, the Born-radius workspace and the ScoreCard, then launchNonbonded and
//       launchValence with EvaluateForce::YES, EvaluateEnergy::YES).  Three untimed steps, then
//       <evals> steps timed with CUDA events on the default stream, which STORMM launches on.
//       Prints "evals=<n> ms=<total> systems=<m> atoms=<a>".  With --out, writes the per-term
//       energies of every system and the forces of the last step.
//   minimize <list-file> <out.bin> --maxcyc N --ncyc N [--ntpr N] [--prec single|double]
//            [--cdcyc N --clash-r0 X --clash-ratio X]
//       STORMM's launchMinimization (MolecularMechanics/hpc_minimization.h:138) over the
//       synthesis, the first --cdcyc cycles clash-damped.  Prints "minimize ms=<wall>
//       systems=<m>" (the whole call, host setup included) and writes each system's
//       starting coordinates (as the synthesis holds them, on its fixed-point grid),
//       potential-energy history (one sample every ntpr cycles, ntpr defaulting to 1), final
//       per-term energies and final coordinates.
//
// Options: --igb {1,2,5,7,8} (default 5 = OBC-II), --diel X (80).  Topologies are read as the CPU
// driver reads them (radius set NONE, so that the radii written in the prmtop are used).
#include <cuda_runtime.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>
#include "copyright.h"
#include "Accelerator/core_kernel_manager.h"
#include "Accelerator/hpc_config.h"
#include "Constants/fixed_precision.h"
#include "Constants/symbol_values.h"
#include "MolecularMechanics/hpc_minimization.h"
#include "MolecularMechanics/mm_controls.h"
#include "Namelists/nml_minimize.h"
#include "Potential/cacheresource.h"
#include "Potential/hpc_nonbonded_potential.h"
#include "Potential/hpc_valence_potential.h"
#include "Potential/scorecard.h"
#include "Synthesis/atomgraph_synthesis.h"
#include "Synthesis/implicit_solvent_workspace.h"
#include "Synthesis/nonbonded_workunit.h"
#include "Synthesis/phasespace_synthesis.h"
#include "Synthesis/static_mask_synthesis.h"
#include "Synthesis/valence_workunit.h"
#include "Topology/atomgraph.h"
#include "Trajectory/phasespace.h"
#include "Trajectory/thermostat.h"

using namespace stormm;
using namespace stormm::card;
using namespace stormm::energy;
using namespace stormm::mm;
using namespace stormm::namelist;
using namespace stormm::synthesis;
using namespace stormm::topology;
using namespace stormm::trajectory;

namespace {

struct Options {
  int igb = 5;
  double diel = 80.0;
  PrecisionModel prec = PrecisionModel::SINGLE;
  std::string out;
  int maxcyc = 0;
  int ncyc = 0;
  int ntpr = 1;
  int cdcyc = 0;
  double clash_r0 = -1.0;
  double clash_ratio = -1.0;
};

// Record file: for each record, int32 name length, name bytes, one dtype char ('d' double,
// 'i' int32), int64 element count, raw little-endian data (the CPU driver's format).
class RecordWriter {
public:
  explicit RecordWriter(const std::string &path) : out_(path, std::ios::binary) {
    if (!out_) {
      std::fprintf(stderr, "cannot open %s\n", path.c_str());
      std::exit(2);
    }
  }
  template <typename T> void put(const std::string &name, char dtype, const T* data, size_t n) {
    const int32_t len = name.size();
    out_.write(reinterpret_cast<const char*>(&len), 4);
    out_.write(name.data(), len);
    out_.write(&dtype, 1);
    const int64_t cnt = n;
    out_.write(reinterpret_cast<const char*>(&cnt), 8);
    if (n > 0) {
      out_.write(reinterpret_cast<const char*>(data), n * sizeof(T));
    }
  }
  void d(const std::string &name, const std::vector<double> &v) { put(name, 'd', v.data(), v.size()); }
  void i(const std::string &name, const std::vector<int> &v) { put(name, 'i', v.data(), v.size()); }
private:
  std::ofstream out_;
};

const std::vector<StateVariable> kTerms = {
  StateVariable::BOND, StateVariable::ANGLE, StateVariable::PROPER_DIHEDRAL,
  StateVariable::IMPROPER_DIHEDRAL, StateVariable::VDW, StateVariable::VDW_ONE_FOUR,
  StateVariable::ELECTROSTATIC, StateVariable::ELEC_ONE_FOUR, StateVariable::GENERALIZED_BORN
};

ImplicitSolventModel igbModel(int igb) {
  switch (igb) {
  case 1: return ImplicitSolventModel::HCT_GB;
  case 2: return ImplicitSolventModel::OBC_GB;
  case 5: return ImplicitSolventModel::OBC_GB_II;
  case 7: return ImplicitSolventModel::NECK_GB;
  case 8: return ImplicitSolventModel::NECK_GB_II;
  default:
    std::fprintf(stderr, "unsupported igb %d\n", igb);
    std::exit(2);
  }
}

// The systems of a list file, each with its own topology
struct SystemList {
  std::vector<AtomGraph> ags;
  std::vector<PhaseSpace> pss;
  std::vector<AtomGraph*> ag_ptrs;
  std::vector<int> indices;
  long long atoms = 0;
};

void readSystems(const std::string &list_file, const Options &opt, SystemList *sl) {
  std::ifstream lst(list_file);
  std::string top, crd;
  std::vector<std::string> tops, crds;
  while (lst >> top >> crd) {
    tops.push_back(top);
    crds.push_back(crd);
  }
  if (tops.empty()) {
    std::fprintf(stderr, "no systems listed in %s\n", list_file.c_str());
    std::exit(2);
  }
  sl->ags.resize(tops.size());
  for (size_t k = 0; k < tops.size(); k++) {
    sl->ags[k].buildFromPrmtop(tops[k], ExceptionResponse::SILENT, symbols::amber_ancient_bioq,
                               1.2, 2.0, default_charge_rounding_tol,
                               default_charge_precision_inc);
    sl->ags[k].setImplicitSolventModel(igbModel(opt.igb), opt.diel, 0.0, AtomicRadiusSet::NONE,
                                       ExceptionResponse::SILENT);
    sl->pss.emplace_back(crds[k], CoordinateFileKind::AMBER_INPCRD);
    sl->atoms += sl->ags[k].getAtomCount();
  }
  for (size_t k = 0; k < tops.size(); k++) {
    sl->ag_ptrs.push_back(&sl->ags[k]);
    sl->indices.push_back(static_cast<int>(k));
  }
}

void check(cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(err));
    std::exit(3);
  }
}

void putCoordinates(RecordWriter *rw, const std::string &name, const PhaseSpaceSynthesis &ps,
                    int nsys, bool forces) {
  std::vector<double> c;
  for (int i = 0; i < nsys; i++) {
    const PhaseSpace p = ps.exportSystem(i, HybridTargetLevel::HOST);
    const PhaseSpaceReader r = p.data();
    for (int j = 0; j < r.natom; j++) {
      c.push_back(forces ? r.xfrc[j] : r.xcrd[j]);
      c.push_back(forces ? r.yfrc[j] : r.ycrd[j]);
      c.push_back(forces ? r.zfrc[j] : r.zcrd[j]);
    }
  }
  rw->d(name, c);
}

void putTerms(RecordWriter *rw, const std::string &name, const ScoreCard &sc, int nsys) {
  std::vector<double> e;
  for (int i = 0; i < nsys; i++) {
    for (StateVariable sv : kTerms) {
      e.push_back(sc.reportInstantaneousStates(sv, i));
    }
  }
  rw->d(name, e);
}

int runTime(const std::string &list_file, int evals, const Options &opt) {
  const HpcConfig gpu_config(ExceptionResponse::WARN);
  const std::vector<int> my_gpus = gpu_config.getGpuDevice(1);
  const GpuDetails gpu = gpu_config.getGpuInfo(my_gpus[0]);
  SystemList sl;
  readSystems(list_file, opt, &sl);
  AtomGraphSynthesis poly_ag(sl.ag_ptrs, sl.indices, ExceptionResponse::WARN, gpu);
  StaticExclusionMaskSynthesis poly_se(poly_ag.getUniqueTopologies(),
                                       poly_ag.getTopologyIndices());
  poly_ag.loadNonbondedWorkUnits(poly_se);
  PhaseSpaceSynthesis poly_ps(sl.pss, sl.ag_ptrs);
  const CoreKlManager launcher(gpu, poly_ag);
  poly_ag.upload();
  poly_se.upload();
  poly_ps.upload();
  const int nsys = poly_ag.getSystemCount();
  const int2 vale_lp = launcher.getValenceKernelDims(opt.prec, EvaluateForce::YES,
                                                     EvaluateEnergy::YES,
                                                     AccumulationMethod::SPLIT,
                                                     VwuGoal::ACCUMULATE, ClashResponse::NONE);
  const int2 nonb_lp = launcher.getNonbondedKernelDims(opt.prec, poly_ag.getNonbondedWorkType(),
                                                       EvaluateForce::YES, EvaluateEnergy::YES,
                                                       AccumulationMethod::SPLIT,
                                                       poly_ag.getImplicitSolventModel(),
                                                       ClashResponse::NONE);
  CacheResource vale_cache(vale_lp.x, maximum_valence_work_unit_atoms);
  CacheResource nonb_cache(nonb_lp.x, small_block_max_atoms);
  ImplicitSolventWorkspace ism_space(poly_ag.getSystemAtomOffsets(),
                                     poly_ag.getSystemAtomCounts(), opt.prec);
  Thermostat heat_bath(poly_ag, ThermostatKind::NONE);
  ScoreCard sc(nsys, 1, default_energy_scale_bits);
  MolecularMechanicsControls mmctrl;
  mmctrl.primeWorkUnitCounters(launcher, EvaluateForce::YES, EvaluateEnergy::YES,
                               VwuGoal::ACCUMULATE, opt.prec, opt.prec, poly_ag);
  const HybridTargetLevel devc = HybridTargetLevel::DEVICE;
  auto step = [&]() {
    poly_ps.initializeForces(gpu, devc);
    ism_space.initialize(devc, CoordinateCycle::WHITE, gpu);
    sc.initialize(devc, gpu);
    launchNonbonded(opt.prec, poly_ag, poly_se, &mmctrl, &poly_ps, &heat_bath, &sc, &nonb_cache,
                    &ism_space, EvaluateForce::YES, EvaluateEnergy::YES, AccumulationMethod::SPLIT,
                    launcher);
    launchValence(opt.prec, poly_ag, &mmctrl, &poly_ps, &heat_bath, &sc, &vale_cache,
                  EvaluateForce::YES, EvaluateEnergy::YES, VwuGoal::ACCUMULATE,
                  AccumulationMethod::SPLIT, launcher);
    mmctrl.incrementStep();
  };
  for (int k = 0; k < 3; k++) {
    step();
  }
  check(cudaDeviceSynchronize(), "warm-up");
  cudaEvent_t t0, t1;
  check(cudaEventCreate(&t0), "event");
  check(cudaEventCreate(&t1), "event");
  check(cudaEventRecord(t0, 0), "event record");
  for (int k = 0; k < evals; k++) {
    step();
  }
  check(cudaEventRecord(t1, 0), "event record");
  check(cudaEventSynchronize(t1), "timed steps");
  float ms = 0.0f;
  check(cudaEventElapsedTime(&ms, t0, t1), "elapsed");
  std::printf("evals=%d ms=%.6f systems=%d atoms=%lld\n", evals, ms, nsys, sl.atoms);
  if (!opt.out.empty()) {
    sc.commit(devc, gpu);
    sc.incrementSampleCount();
    sc.download();
    poly_ps.download();
    RecordWriter rw(opt.out);
    putTerms(&rw, "energy_terms", sc, nsys);
    putCoordinates(&rw, "forces", poly_ps, nsys, true);
  }
  return 0;
}

int runMinimize(const std::string &list_file, const Options &opt) {
  const HpcConfig gpu_config(ExceptionResponse::WARN);
  const std::vector<int> my_gpus = gpu_config.getGpuDevice(1);
  const GpuDetails gpu = gpu_config.getGpuInfo(my_gpus[0]);
  SystemList sl;
  readSystems(list_file, opt, &sl);
  AtomGraphSynthesis poly_ag(sl.ag_ptrs, sl.indices, ExceptionResponse::WARN, gpu);
  StaticExclusionMaskSynthesis poly_se(poly_ag.getUniqueTopologies(),
                                       poly_ag.getTopologyIndices());
  poly_ag.loadNonbondedWorkUnits(poly_se);
  PhaseSpaceSynthesis poly_ps(sl.pss, sl.ag_ptrs);
  poly_ag.upload();
  poly_se.upload();
  poly_ps.upload();
  const int nsys = poly_ag.getSystemCount();
  std::vector<double> start_coords;
  for (int i = 0; i < nsys; i++) {
    const PhaseSpace p = poly_ps.exportSystem(i, HybridTargetLevel::HOST);
    const PhaseSpaceReader r = p.data();
    for (int j = 0; j < r.natom; j++) {
      start_coords.push_back(r.xcrd[j]);
      start_coords.push_back(r.ycrd[j]);
      start_coords.push_back(r.zcrd[j]);
    }
  }
  MinimizeControls mincon;
  mincon.setTotalCycles(opt.maxcyc);
  mincon.setSteepestDescentCycles(opt.ncyc);
  mincon.setClashDampingCycles(opt.cdcyc);
  if (opt.clash_r0 >= 0.0) {
    mincon.setAbsoluteClashDistance(opt.clash_r0);
  }
  if (opt.clash_ratio >= 0.0) {
    mincon.setVdwClashRatio(opt.clash_ratio);
  }
  mincon.setDiagnosticPrintFrequency(opt.ntpr);
  check(cudaDeviceSynchronize(), "upload");
  const auto w0 = std::chrono::steady_clock::now();
  ScoreCard sc = launchMinimization(poly_ag, poly_se, &poly_ps, mincon, gpu, opt.prec,
                                    default_energy_scale_bits);
  check(cudaDeviceSynchronize(), "minimization");
  const double ms =
    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
  std::printf("minimize ms=%.6f systems=%d atoms=%lld cycles=%d\n", ms, nsys, sl.atoms,
              opt.maxcyc);
  sc.download();
  poly_ps.download();
  RecordWriter rw(opt.out);
  std::vector<double> hist;
  std::vector<int> hist_len;
  for (int i = 0; i < nsys; i++) {
    // the potential energy of each sample is the sum of the terms' histories (the GPU
    // minimizer commits the terms; the potential energy is not a state of its own there)
    std::vector<double> h;
    for (StateVariable sv : kTerms) {
      const std::vector<double> t = sc.reportHistory(sv, i);
      if (h.empty()) {
        h.assign(t.size(), 0.0);
      }
      for (size_t k = 0; k < t.size() && k < h.size(); k++) {
        h[k] += t[k];
      }
    }
    hist.insert(hist.end(), h.begin(), h.end());
    hist_len.push_back(static_cast<int>(h.size()));
  }
  rw.d("min_start_coords", start_coords);
  rw.d("min_potential_history", hist);
  rw.i("min_history_length", hist_len);
  putTerms(&rw, "min_final_terms", sc, nsys);
  putCoordinates(&rw, "min_final_coords", poly_ps, nsys, false);
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s time|minimize ...\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  std::vector<std::string> pos;
  Options opt;
  for (int k = 2; k < argc; k++) {
    const std::string a = argv[k];
    auto next = [&]() -> std::string {
      if (k + 1 >= argc) {
        std::fprintf(stderr, "%s needs a value\n", a.c_str());
        std::exit(2);
      }
      return std::string(argv[++k]);
    };
    if (a == "--igb") opt.igb = std::stoi(next());
    else if (a == "--diel") opt.diel = std::stod(next());
    else if (a == "--prec") {
      const std::string p = next();
      opt.prec = (p == "double") ? PrecisionModel::DOUBLE : PrecisionModel::SINGLE;
    }
    else if (a == "--out") opt.out = next();
    else if (a == "--maxcyc") opt.maxcyc = std::stoi(next());
    else if (a == "--ncyc") opt.ncyc = std::stoi(next());
    else if (a == "--ntpr") opt.ntpr = std::stoi(next());
    else if (a == "--cdcyc") opt.cdcyc = std::stoi(next());
    else if (a == "--clash-r0") opt.clash_r0 = std::stod(next());
    else if (a == "--clash-ratio") opt.clash_ratio = std::stod(next());
    else pos.push_back(a);
  }
  if (mode == "time" && pos.size() == 2) {
    return runTime(pos[0], std::stoi(pos[1]), opt);
  }
  if (mode == "minimize" && pos.size() == 2) {
    opt.out = pos[1];
    return runMinimize(pos[0], opt);
  }
  std::fprintf(stderr, "bad arguments for mode %s\n", mode.c_str());
  return 2;
}
