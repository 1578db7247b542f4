// Drives the STORMM-named C++ layer (include/stormm_b200.hpp) the way a STORMM caller would:
// topologies and coordinates from Amber files, a synthesis, launchValence + launchNonbonded into
// a ScoreCard, then launchMinimization.  Results are written as text ("name count values...",
// 17 significant digits) for the Python tests to compare with the library's Python path and the
// oracle.
//
//   launcher_check host <out> <prmtop> <inpcrd>    host-side checks (no device needed): reading,
//                                                  synthesis set-up, error behaviour
//   launcher_check device <out> <prmtop> <inpcrd> [<prmtop> <inpcrd> ...]
//                                                  every system twice (topologies reused)
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "stormm_b200.hpp"

using namespace stormm_b200;

namespace {

void put(FILE* f, const std::string &name, const std::vector<double> &v) {
  std::fprintf(f, "%s %zu", name.c_str(), v.size());
  for (double x : v) {
    std::fprintf(f, " %.17g", x);
  }
  std::fprintf(f, "\n");
}

template <typename F> bool throwsRuntimeError(F &&f, const char* fragment, FILE* out,
                                              const char* label) {
  try {
    f();
  }
  catch (const std::runtime_error &e) {
    const bool ok = std::string(e.what()).find(fragment) != std::string::npos;
    std::fprintf(out, "error %s %d %s\n", label, ok ? 1 : 0, e.what());
    return ok;
  }
  std::fprintf(out, "error %s 0 (nothing thrown)\n", label);
  return false;
}

int hostChecks(FILE* out, const std::string &top, const std::string &crd) {
  AtomGraph ag(top);
  PhaseSpace ps(crd);
  std::fprintf(out, "atoms 1 %d\n", ag.getAtomCount());
  put(out, "coords", ps.getInterlacedCoordinates());
  AtomGraphSynthesis poly_ag({&ag}, {0, 0});
  poly_ag.setImplicitSolventModel(ImplicitSolventModel::OBC_GB_II);
  PhaseSpaceSynthesis poly_ps({ps, ps}, {&ag, &ag});
  std::fprintf(out, "systems 1 %d\n", poly_ps.getSystemCount());
  StaticExclusionMaskSynthesis poly_se(poly_ag);
  poly_ag.loadNonbondedWorkUnits(poly_se, InitializationTask::GB_MINIMIZATION);
  const std::vector<int> &abstracts = poly_ag.getNonbondedWorkUnitAbstracts();
  const std::vector<uint32_t> &insr = poly_ag.getNonbondedWorkUnitInstructions();
  put(out, "nbwu_abstracts", std::vector<double>(abstracts.begin(), abstracts.end()));
  put(out, "nbwu_insr", std::vector<double>(insr.begin(), insr.end()));
  bool ok = true;
  ok &= throwsRuntimeError([&]() { AtomGraph missing(top + ".absent"); }, "cannot open", out,
                           "missing_file");
  ok &= throwsRuntimeError([&]() { ScoreCard sc(0); }, "at least one system", out,
                           "empty_scorecard");
  ok &= throwsRuntimeError([&]() { AtomGraphSynthesis bad({&ag}, {1}); }, "out of range", out,
                           "topology_index");
  ok &= throwsRuntimeError(
      [&]() {
        ScoreCard sc(2);
        CoreKlManager launcher;
        MolecularMechanicsControls mmctrl;
        Thermostat heat_bath;
        CacheResource tb_space;
        launchValence(PrecisionModel::SINGLE, poly_ag, &mmctrl, &poly_ps, &heat_bath, &sc,
                      &tb_space, EvaluateForce::YES, EvaluateEnergy::YES, VwuGoal::ACCUMULATE,
                      launcher);
      },
      "upload() has not been called", out, "launch_before_upload");
  ok &= throwsRuntimeError([&]() { MinimizeControls m; m.setTotalCycles(0); }, "positive", out,
                           "minimize_controls");
  // Without a device the upload itself fails with the library's message
  try {
    poly_ag.upload();
    std::fprintf(out, "upload 1 1\n");
  }
  catch (const std::runtime_error &e) {
    std::fprintf(out, "upload 1 0 %s\n", e.what());
  }
  return ok ? 0 : 1;
}

int deviceChecks(FILE* out, const std::vector<std::string> &files) {
  std::vector<AtomGraph> graphs;
  std::vector<PhaseSpace> coords;
  graphs.reserve(files.size() / 2);
  for (size_t k = 0; k + 1 < files.size(); k += 2) {
    graphs.emplace_back(files[k]);
    coords.emplace_back(files[k + 1]);
  }
  const int ntop = static_cast<int>(graphs.size());
  std::vector<AtomGraph*> ag_list;
  for (AtomGraph &ag : graphs) {
    ag_list.push_back(&ag);
  }
  std::vector<int> systems;
  for (int rep = 0; rep < 2; rep++) {
    for (int t = 0; t < ntop; t++) {
      systems.push_back(t);
    }
  }
  AtomGraphSynthesis poly_ag(ag_list, systems);
  poly_ag.setImplicitSolventModel(ImplicitSolventModel::OBC_GB_II);
  PhaseSpaceSynthesis poly_ps(coords, ag_list, systems);
  StaticExclusionMaskSynthesis poly_se(poly_ag);
  poly_ag.upload();
  poly_ps.upload();
  const int nsys = poly_ag.getSystemCount();

  // One force + energy evaluation: valence, then nonbonded + GB
  ScoreCard sc(nsys);
  ImplicitSolventWorkspace ism_space(poly_ag);
  MolecularMechanicsControls mmctrl;
  Thermostat heat_bath;
  CacheResource tb_space;
  GpuDetails gpu;
  CoreKlManager launcher(gpu, poly_ag);
  sc.initialize();
  ism_space.initialize();
  poly_ps.initializeForces();
  launchValence(PrecisionModel::SINGLE, poly_ag, &mmctrl, &poly_ps, &heat_bath, &sc, &tb_space,
                EvaluateForce::YES, EvaluateEnergy::YES, VwuGoal::ACCUMULATE, launcher);
  launchNonbonded(PrecisionModel::SINGLE, poly_ag, poly_se, &mmctrl, &poly_ps, &heat_bath, &sc,
                  &tb_space, &ism_space, EvaluateForce::YES, EvaluateEnergy::YES, launcher);
  sc.download();
  poly_ps.download();
  ism_space.download();
  std::vector<double> energies, forces;
  for (int s = 0; s < nsys; s++) {
    for (int v = 0; v < SB_NRG_STRIDE; v++) {
      energies.push_back(sc.reportInstantaneousStates(static_cast<StateVariable>(v), s));
    }
    const std::vector<double> f = poly_ps.getInterlacedCoordinates(s, TrajectoryKind::FORCES);
    forces.insert(forces.end(), f.begin(), f.end());
  }
  put(out, "energies", energies);
  put(out, "potential", sc.reportPotentialEnergies());
  put(out, "forces", forces);
  put(out, "psi", ism_space.getPsi());
  put(out, "radii", ism_space.getEffectiveRadii());

  // An energy-only, clash-damped nonbonded evaluation into a second ScoreCard
  ScoreCard sc_clash(nsys);
  sc_clash.initialize();
  launchNonbonded(PrecisionModel::SINGLE, poly_ag, poly_se, &mmctrl, &poly_ps, &heat_bath,
                  &sc_clash, &tb_space, &ism_space, EvaluateForce::NO, EvaluateEnergy::YES,
                  launcher, 0.5, 0.8);
  sc_clash.download();
  std::vector<double> clash;
  for (int s = 0; s < nsys; s++) {
    for (int v = 0; v < SB_NRG_STRIDE; v++) {
      clash.push_back(sc_clash.reportInstantaneousStates(static_cast<StateVariable>(v), s));
    }
  }
  put(out, "clash_energies", clash);

  // Minimization from the file coordinates
  poly_ps.upload();
  MinimizeControls mincon;
  mincon.setTotalCycles(40);
  mincon.setSteepestDescentCycles(10);
  mincon.setClashDampingCycles(5);
  mincon.setDiagnosticPrintFrequency(10);
  ScoreCard result = launchMinimization(poly_ag, poly_se, &poly_ps, mincon, gpu);
  poly_ps.download();
  put(out, "min_potential", result.reportPotentialEnergies());
  std::vector<double> hist, xyz;
  for (int s = 0; s < nsys; s++) {
    const std::vector<double> h = result.reportHistory(s);
    hist.insert(hist.end(), h.begin(), h.end());
    const std::vector<double> c = poly_ps.getInterlacedCoordinates(s);
    xyz.insert(xyz.end(), c.begin(), c.end());
  }
  put(out, "min_history", hist);
  put(out, "min_coords", xyz);

  // A line search driven step by step, as STORMM's launchMinimization drives its kernels:
  // evaluations by launchValence + launchNonbonded, launchConjugateGradient after the line-start
  // evaluation, launchLineAdvance after each of the four evaluations (no clash-damped cycles)
  poly_ps.upload();
  MinimizeControls step_con;
  step_con.setTotalCycles(12);
  step_con.setSteepestDescentCycles(4);
  step_con.setClashDampingCycles(0);
  MolecularMechanicsControls step_ctrl(step_con);
  LineMinimization line_record(nsys, step_con.getInitialStep());
  ReductionBridge rbg(static_cast<size_t>(nsys));
  ScoreCard sc_steps(nsys);
  for (int cyc = 0; cyc < step_con.getTotalCycles(); cyc++) {
    for (int move = 0; move < 4; move++) {
      const EvaluateForce ef = (move == 0) ? EvaluateForce::YES : EvaluateForce::NO;
      sc_steps.initialize();
      if (move == 0) {
        poly_ps.initializeForces();
      }
      launchValence(PrecisionModel::SINGLE, poly_ag, &step_ctrl, &poly_ps, &heat_bath, &sc_steps,
                    &tb_space, ef, EvaluateEnergy::YES, VwuGoal::ACCUMULATE, launcher);
      launchNonbonded(PrecisionModel::SINGLE, poly_ag, poly_se, &step_ctrl, &poly_ps, &heat_bath,
                      &sc_steps, &tb_space, &ism_space, ef, EvaluateEnergy::YES, launcher);
      if (move == 0) {
        launchConjugateGradient(PrecisionModel::SINGLE, poly_ag, &poly_ps, &rbg, &step_ctrl,
                                launcher);
      }
      launchLineAdvance(PrecisionModel::SINGLE, &poly_ps, poly_ag, &sc_steps, &line_record, move,
                        launcher);
    }
  }
  poly_ps.download();
  std::vector<double> step_xyz;
  for (int s = 0; s < nsys; s++) {
    const std::vector<double> c = poly_ps.getInterlacedCoordinates(s);
    step_xyz.insert(step_xyz.end(), c.begin(), c.end());
  }
  put(out, "steps_coords", step_xyz);

  // The same minimization with PrecisionModel::DOUBLE on a synthesis uploaded for FP64
  AtomGraphSynthesis poly_ag64(ag_list, systems);
  poly_ag64.setImplicitSolventModel(ImplicitSolventModel::OBC_GB_II);
  PhaseSpaceSynthesis poly_ps64(coords, ag_list, systems);
  StaticExclusionMaskSynthesis poly_se64(poly_ag64);
  poly_ag64.upload(PrecisionModel::DOUBLE);
  poly_ps64.upload();
  ScoreCard result64 = launchMinimization(poly_ag64, poly_se64, &poly_ps64, mincon, gpu,
                                          PrecisionModel::DOUBLE);
  poly_ps64.download();
  std::vector<double> xyz64;
  for (int s = 0; s < nsys; s++) {
    const std::vector<double> c = poly_ps64.getInterlacedCoordinates(s);
    xyz64.insert(xyz64.end(), c.begin(), c.end());
  }
  put(out, "min64_potential", result64.reportPotentialEnergies());
  put(out, "min64_coords", xyz64);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5 || (argc % 2) == 0) {
    std::fprintf(stderr, "usage: %s host|device <out> <prmtop> <inpcrd> [...]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  FILE* out = std::fopen(argv[2], "w");
  if (out == nullptr) {
    std::fprintf(stderr, "cannot write %s\n", argv[2]);
    return 2;
  }
  int rc = 2;
  try {
    if (mode == "host") {
      rc = hostChecks(out, argv[3], argv[4]);
    }
    else if (mode == "device") {
      rc = deviceChecks(out, std::vector<std::string>(argv + 3, argv + argc));
    }
  }
  catch (const std::exception &e) {
    std::fprintf(stderr, "launcher_check: %s\n", e.what());
    rc = 1;
  }
  std::fclose(out);
  return rc;
}
