// Driver over STORMM's own CPU library (built from the reference sources by the Makefile beside
// this file).  It is test infrastructure only: it reads Amber prmtop / inpcrd files through
// STORMM's AtomGraph and PhaseSpace, runs STORMM's FP64 CPU evaluators, and writes what it
// computed to a small binary record file that tests/golden/make_golden.py turns into fixtures.
// It also times the evaluators for the CPU baseline.
//
// Modes:
//   eval <prmtop> <inpcrd> <out.bin> [options]
//       Parameters as STORMM parsed them, FP64 energies per term (double sums and the ScoreCard's
//       fixed-point sums), per-term forces, GB intermediates (psi, effective radii, sumdeijda)
//       and the StaticExclusionMask tables.
//   minimize <prmtop> <inpcrd> <out.bin> --maxcyc N --ncyc N [options]
//       STORMM's CPU line minimizer (MolecularMechanics/minimization.h:157); writes the energy
//       history and the final coordinates.  --cdcyc N runs its first N cycles clash-damped with
//       --clash-r0 / --clash-ratio (STORMM defaults 0.2 A and 0.5).
//   time <list-file> <seconds> [options]
//       Evaluates energy + forces (evalRestrainedMMGB) over the systems named in <list-file>
//       (one "prmtop inpcrd" pair per line) round-robin until <seconds> of wall time pass, and
//       prints "evals=<n> seconds=<t>".  With --minimize N it instead runs N-cycle minimizations
//       and prints "minimizations=<n> seconds=<t>".
//
//   sdf <file> <out.bin>
//       STORMM's MdlMol parse of each compound of an SD / MOL file (readStructureDataFile).
//   geometry <prmtop> <list-file> <out.bin>
//       STORMM's clash verdict (detectClash) for each coordinate file listed and its
//       mass-weighted aligned RMSD (RMSDMethod::ALIGN_MASS) against the first.
//   writecrd <in.inpcrd> <out.inpcrd>
//       The coordinates of an Amber input-coordinate file written back by STORMM's
//       PhaseSpace::exportToFile (CoordinateFileKind::AMBER_INPCRD).
//
//   vwu <prmtop> <out.bin> [--vwu-atoms N]
//       STORMM's valence work units of one topology (Synthesis/valence_workunit.cpp,
//       buildValenceWorkUnits with a blank RestraintApparatus and an atom limit of N, default
//       the synthesis sizing for one copy on 148 SMs): the ValenceKit arrays they are built from
//       and, per unit, the import / update lists, manipulation masks, task counts, term lists,
//       energy-accumulation masks and the instructions stored against the topology's own
//       parameter indices.
//   vwusize <counts-file> <sm-count> <out.bin>
//       calculateValenceWorkUnitSize over each line of atom counts (one synthesis per line):
//       the atom limit and kernel width it picks for that many SMs (sm-count 0: the overload
//       without an SM count).
//   restraint <prmtop> <inpcrd> <restraint-file> <out.bin>
//       STORMM's restraint evaluation (evaluateRestraints, Potential/valence_potential.tpp:
//       1558-2050) for constant restraints listed one a line: "kind i j k l k2 k3 r1 r2 r3 r4 x
//       y z" (kind 1 positional, 2 distance, 3 angle, 4 dihedral; 0-based atoms, unused ones
//       -1; the target x y z used by positional restraints); writes each restraint's energy,
//       the total and the forces.
//   restraintramp <prmtop> <inpcrd> <restraint-file> <steps> <out.bin>
//       The same for time-dependent restraints, one a line: "kind i j k l init_step final_step
//       k2 k3 r1 r2 r3 r4 x y z k2' k3' r1' r2' r3' r4' x' y' z'" (initial values, then final
//       ones), evaluated at each step of the comma-separated <steps>: each restraint's energy,
//       the total and the forces at step s are written as restraint_energies_s,
//       restraint_total_s and frc_restraint_s.
//   sasa <prmtop> <inpcrd> <n-points> <out.bin>
//       STORMM's surface area (Potential/surface_area.cpp:46-99, LJ-sigma radii, every
//       molecule, probe 1.4 A, double precision): the sphere points it places, the area
//       (weight 1) and the energy at the default 0.005 kcal/mol per A^2.
//   nbwu <list-file> <out.bin> [--init-task N]
//       STORMM's nonbonded work units (Synthesis/nonbonded_workunit.cpp) for a synthesis: each
//       line of <list-file> is "<prmtop> <system count>", the systems laid out topology by
//       topology; writes the StaticExclusionMaskSynthesis tables and the abstracts and tile
//       instructions AtomGraphSynthesis::loadNonbondedWorkUnits stores (InitializationTask N,
//       default 3 = GB_MINIMIZATION).
//
// Options: --igb {0,1,2,5,7,8} (default 5 = OBC-II), --diel X (80), --salt X (0),
//          --qtol X --qdisc X (charge smoothing, STORMM defaults), --scee X --scnb X,
//          --quantize (round coordinates to the 2^-32 Angstrom fixed-point grid first).
//          In eval mode, --clash-r0 X and --clash-ratio X add the clash-mitigated evaluation
//          (softened Coulomb and Lennard-Jones cores, Potential/soft_core_potentials.tpp) of the
//          MM driver as the records clash_frc_total and clash_energy_terms.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "copyright.h"
#include "Constants/generalized_born.h"
#include "Constants/symbol_values.h"
#include "MoleculeFormat/mdlmol.h"
#include "MolecularMechanics/minimization.h"
#include "MolecularMechanics/mm_evaluation.h"
#include "Namelists/nml_minimize.h"
#include "Potential/nonbonded_potential.h"
#include "Potential/scorecard.h"
#include "Potential/static_exclusionmask.h"
#include "Potential/valence_potential.h"
#include "Potential/surface_area.h"
#include "Math/geodesic.h"
#include "Math/series_ops.h"
#include "Restraints/bounded_restraint.h"
#include "Restraints/restraint_apparatus.h"
#include "Structure/clash_detection.h"
#include "Structure/rmsd.h"
#include "Trajectory/coordinateframe.h"
#include "Synthesis/atomgraph_synthesis.h"
#include "Synthesis/static_mask_synthesis.h"
#include "Synthesis/synthesis_abstracts.h"
#include "Synthesis/valence_workunit.h"
#include "Topology/atomgraph.h"
#include "Trajectory/phasespace.h"
#include "Trajectory/trajectory_enumerators.h"

using namespace stormm;
using namespace stormm::energy;
using namespace stormm::topology;
using namespace stormm::trajectory;
using namespace stormm::restraints;
using namespace stormm::namelist;
using namespace stormm::mm;
using stormm::generalized_born_defaults::NeckGeneralizedBornTable;
using stormm::generalized_born_defaults::NeckGeneralizedBornKit;

namespace {

struct Options {
  int igb = 5;
  double diel = 80.0;
  double salt = 0.0;
  double qtol = -1.0;
  double qdisc = -1.0;
  double scee = 1.2;
  double scnb = 2.0;
  bool quantize = false;
  int maxcyc = 0;
  int ncyc = 0;
  int minimize_cycles = 0;
  double dx0 = 0.01;
  int cdcyc = 0;
  double clash_r0 = -1.0;
  double clash_ratio = -1.0;
};

// Record file: for each record, int32 name length, name bytes, one dtype char ('d' double,
// 'i' int32, 'q' int64, 'u' uint32), int64 element count, raw little-endian data.
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
  void d(const std::string &name, const double* p, size_t n) { put(name, 'd', p, n); }
  void i(const std::string &name, const std::vector<int> &v) { put(name, 'i', v.data(), v.size()); }
  void i(const std::string &name, const int* p, size_t n) { put(name, 'i', p, n); }
  void u(const std::string &name, const uint* p, size_t n) { put(name, 'u', p, n); }
  void scalar(const std::string &name, double v) { put(name, 'd', &v, 1); }
  void iscalar(const std::string &name, int v) { put(name, 'i', &v, 1); }
private:
  std::ofstream out_;
};

ImplicitSolventModel igbModel(int igb) {
  switch (igb) {
  case 0: return ImplicitSolventModel::NONE;
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

AtomGraph loadTopology(const std::string &prmtop, const Options &opt) {
  AtomGraph ag;
  const double qtol = (opt.qtol >= 0.0) ? opt.qtol : default_charge_rounding_tol;
  const double qdisc = (opt.qdisc >= 0.0) ? opt.qdisc : default_charge_precision_inc;
  ag.buildFromPrmtop(prmtop, ExceptionResponse::SILENT, symbols::amber_ancient_bioq, opt.scee,
                     opt.scnb, qtol, qdisc);
  ag.setImplicitSolventModel(igbModel(opt.igb), opt.diel, opt.salt, AtomicRadiusSet::NONE,
                             ExceptionResponse::SILENT);
  return ag;
}

void quantizeCoordinates(PhaseSpace *ps) {
  PhaseSpaceWriter psw = ps->data();
  const double scale = 4294967296.0;
  for (int i = 0; i < psw.natom; i++) {
    psw.xcrd[i] = static_cast<double>(std::llround(psw.xcrd[i] * scale)) / scale;
    psw.ycrd[i] = static_cast<double>(std::llround(psw.ycrd[i] * scale)) / scale;
    psw.zcrd[i] = static_cast<double>(std::llround(psw.zcrd[i] * scale)) / scale;
  }
}

void zeroForces(PhaseSpaceWriter psw) {
  for (int i = 0; i < psw.natom; i++) {
    psw.xfrc[i] = 0.0;
    psw.yfrc[i] = 0.0;
    psw.zfrc[i] = 0.0;
  }
}

void putForces(RecordWriter *rw, const std::string &name, const PhaseSpaceWriter &psw) {
  std::vector<double> f(3 * psw.natom);
  for (int i = 0; i < psw.natom; i++) {
    f[3 * i] = psw.xfrc[i];
    f[3 * i + 1] = psw.yfrc[i];
    f[3 * i + 2] = psw.zfrc[i];
  }
  rw->d(name, f);
}

void putTopology(RecordWriter *rw, const AtomGraph &ag) {
  const NonbondedKit<double> nbk = ag.getDoublePrecisionNonbondedKit();
  const ValenceKit<double> vk = ag.getDoublePrecisionValenceKit();
  const ImplicitSolventKit<double> isk = ag.getDoublePrecisionImplicitSolventKit();
  const ChemicalDetailsKit cdk = ag.getChemicalDetailsKit();
  const int n = nbk.natom;
  rw->iscalar("natom", n);
  rw->scalar("coulomb_constant", nbk.coulomb_constant);
  rw->d("charge", nbk.charge, n);
  rw->i("lj_idx", nbk.lj_idx, n);
  rw->iscalar("n_lj_types", nbk.n_lj_types);
  const size_t nt2 = static_cast<size_t>(nbk.n_lj_types) * nbk.n_lj_types;
  rw->d("lja", nbk.lja_coeff, nt2);
  rw->d("ljb", nbk.ljb_coeff, nt2);
  rw->d("lja14", nbk.lja_14_coeff, nt2);
  rw->d("ljb14", nbk.ljb_14_coeff, nt2);
  rw->i("z_numbers", cdk.z_numbers, n);
  rw->i("nb11_bounds", nbk.nb11_bounds, n + 1);
  rw->i("nb11x", nbk.nb11x, nbk.nb11_bounds[n]);
  rw->i("nb12_bounds", nbk.nb12_bounds, n + 1);
  rw->i("nb12x", nbk.nb12x, nbk.nb12_bounds[n]);
  rw->i("nb13_bounds", nbk.nb13_bounds, n + 1);
  rw->i("nb13x", nbk.nb13x, nbk.nb13_bounds[n]);
  rw->i("nb14_bounds", nbk.nb14_bounds, n + 1);
  rw->i("nb14x", nbk.nb14x, nbk.nb14_bounds[n]);

  // Valence terms, expanded per term
  std::vector<int> bi(vk.nbond), bj(vk.nbond);
  std::vector<double> bk(vk.nbond), bl(vk.nbond);
  for (int t = 0; t < vk.nbond; t++) {
    bi[t] = vk.bond_i_atoms[t];
    bj[t] = vk.bond_j_atoms[t];
    bk[t] = vk.bond_keq[vk.bond_param_idx[t]];
    bl[t] = std::fabs(vk.bond_leq[vk.bond_param_idx[t]]);
  }
  rw->i("bond_i", bi);
  rw->i("bond_j", bj);
  rw->d("bond_k", bk);
  rw->d("bond_r0", bl);
  std::vector<int> ai(vk.nangl), aj(vk.nangl), ak(vk.nangl);
  std::vector<double> akq(vk.nangl), ath(vk.nangl);
  for (int t = 0; t < vk.nangl; t++) {
    ai[t] = vk.angl_i_atoms[t];
    aj[t] = vk.angl_j_atoms[t];
    ak[t] = vk.angl_k_atoms[t];
    akq[t] = vk.angl_keq[vk.angl_param_idx[t]];
    ath[t] = vk.angl_theta[vk.angl_param_idx[t]];
  }
  rw->i("angl_i", ai);
  rw->i("angl_j", aj);
  rw->i("angl_k", ak);
  rw->d("angl_k_eq", akq);
  rw->d("angl_theta0", ath);
  std::vector<int> di(vk.ndihe), dj(vk.ndihe), dk(vk.ndihe), dl(vk.ndihe), dkind(vk.ndihe);
  std::vector<double> damp(vk.ndihe), dfreq(vk.ndihe), dphi(vk.ndihe), de14(vk.ndihe),
                      dv14(vk.ndihe);
  for (int t = 0; t < vk.ndihe; t++) {
    di[t] = vk.dihe_i_atoms[t];
    dj[t] = vk.dihe_j_atoms[t];
    dk[t] = vk.dihe_k_atoms[t];
    dl[t] = vk.dihe_l_atoms[t];
    const int p = vk.dihe_param_idx[t];
    damp[t] = vk.dihe_amp[p];
    dfreq[t] = vk.dihe_freq[p];
    dphi[t] = vk.dihe_phi[p];
    const int a14 = vk.dihe14_param_idx[t];
    de14[t] = (a14 == 0) ? 0.0 : vk.attn14_elec[a14];
    dv14[t] = (a14 == 0) ? 0.0 : vk.attn14_vdw[a14];
    dkind[t] = static_cast<int>(vk.dihe_modifiers[t].w);
  }
  rw->i("dihe_i", di);
  rw->i("dihe_j", dj);
  rw->i("dihe_k", dk);
  rw->i("dihe_l", dl);
  rw->d("dihe_amp", damp);
  rw->d("dihe_freq", dfreq);
  rw->d("dihe_phase", dphi);
  rw->d("dihe_scee", de14);
  rw->d("dihe_scnb", dv14);
  rw->i("dihe_kind", dkind);
  rw->iscalar("ninfr14", vk.ninfr14);

  // CHARMM terms, expanded per term; CMAP surfaces as STORMM holds them (column-major: the
  // value at phi index j and psi index k is at j + k * dim within the surface)
  std::vector<int> ua(2 * vk.nubrd), ca(4 * vk.ncimp), ma(5 * vk.ncmap), ms(vk.ncmap);
  std::vector<double> uk(vk.nubrd), ul(vk.nubrd), ck(vk.ncimp), cp(vk.ncimp);
  for (int t = 0; t < vk.nubrd; t++) {
    ua[2 * t] = vk.ubrd_i_atoms[t];
    ua[2 * t + 1] = vk.ubrd_k_atoms[t];
    uk[t] = vk.ubrd_keq[vk.ubrd_param_idx[t]];
    ul[t] = vk.ubrd_leq[vk.ubrd_param_idx[t]];
  }
  for (int t = 0; t < vk.ncimp; t++) {
    ca[4 * t] = vk.cimp_i_atoms[t];
    ca[4 * t + 1] = vk.cimp_j_atoms[t];
    ca[4 * t + 2] = vk.cimp_k_atoms[t];
    ca[4 * t + 3] = vk.cimp_l_atoms[t];
    ck[t] = vk.cimp_keq[vk.cimp_param_idx[t]];
    cp[t] = vk.cimp_phi[vk.cimp_param_idx[t]];
  }
  for (int t = 0; t < vk.ncmap; t++) {
    ma[5 * t] = vk.cmap_i_atoms[t];
    ma[5 * t + 1] = vk.cmap_j_atoms[t];
    ma[5 * t + 2] = vk.cmap_k_atoms[t];
    ma[5 * t + 3] = vk.cmap_l_atoms[t];
    ma[5 * t + 4] = vk.cmap_m_atoms[t];
    ms[t] = vk.cmap_surf_idx[t];
  }
  rw->i("ubrd_atoms", ua);
  rw->d("ubrd_keq", uk);
  rw->d("ubrd_leq", ul);
  rw->i("cimp_atoms", ca);
  rw->d("cimp_keq", ck);
  rw->d("cimp_phase", cp);
  rw->i("cmap_atoms", ma);
  rw->i("cmap_surface", ms);
  rw->i("cmap_dims", vk.cmap_dim, vk.ncmap_surf);
  rw->d("cmap_values", vk.cmap_surf, vk.ncmap_surf > 0 ? vk.cmap_surf_bounds[vk.ncmap_surf] : 0);

  // Implicit solvent parameters
  rw->iscalar("igb", static_cast<int>(isk.igb));
  rw->scalar("dielectric", isk.dielectric);
  rw->scalar("saltcon", isk.saltcon);
  rw->d("pb_radii", isk.pb_radii, n);
  rw->d("gb_screen", isk.gb_screen, n);
  rw->d("gb_alpha", isk.gb_alpha, n);
  rw->d("gb_beta", isk.gb_beta, n);
  rw->d("gb_gamma", isk.gb_gamma, n);
  rw->i("neck_gb_idx", isk.neck_gb_idx, n);
}

// The neck GB tables (Constants/generalized_born.h NeckGeneralizedBornTable) and cutoff, which
// the neck models (igb 7, 8) look up by pairs of per-atom neck indices
void putNeckTable(RecordWriter *rw, const NeckGeneralizedBornTable &tab) {
  const NeckGeneralizedBornKit<double> k = tab.dpData();
  rw->iscalar("neck_table_size", k.table_size);
  rw->scalar("neck_cut", k.neck_cut);
  rw->d("neck_max_sep", k.max_separation, static_cast<size_t>(k.table_size) * k.table_size);
  rw->d("neck_max_val", k.max_value, static_cast<size_t>(k.table_size) * k.table_size);
}

void putExclusionMask(RecordWriter *rw, const StaticExclusionMask &se) {
  const StaticExclusionMaskReader ser = se.data();
  const int nst = ser.supertile_stride_count;
  rw->iscalar("se_supertile_stride_count", nst);
  rw->i("se_supertile_map_idx", ser.supertile_map_idx, static_cast<size_t>(nst) * nst);
  const size_t n_uni_st = se.getUniqueSuperTileCount();
  const size_t n_uni_t = se.getUniqueTileCount();
  rw->i("se_tile_map_idx", ser.tile_map_idx, n_uni_st * tiles_per_supertile);
  rw->u("se_mask_data", ser.mask_data, n_uni_t * 2 * tile_length);
}

void putCoordinates(RecordWriter *rw, const std::string &name, const PhaseSpaceWriter &psw) {
  std::vector<double> c(3 * psw.natom);
  for (int i = 0; i < psw.natom; i++) {
    c[3 * i] = psw.xcrd[i];
    c[3 * i + 1] = psw.ycrd[i];
    c[3 * i + 2] = psw.zcrd[i];
  }
  rw->d(name, c);
}

const std::vector<StateVariable> kTerms = {
  StateVariable::BOND, StateVariable::ANGLE, StateVariable::PROPER_DIHEDRAL,
  StateVariable::IMPROPER_DIHEDRAL, StateVariable::VDW, StateVariable::VDW_ONE_FOUR,
  StateVariable::ELECTROSTATIC, StateVariable::ELEC_ONE_FOUR, StateVariable::GENERALIZED_BORN
};

void putScoreCard(RecordWriter *rw, const std::string &name, const ScoreCard &sc) {
  std::vector<double> e;
  for (StateVariable sv : kTerms) {
    e.push_back(sc.reportInstantaneousStates(sv, 0));
  }
  rw->d(name, e);
}

int runEval(const std::string &prmtop, const std::string &inpcrd, const std::string &out,
            const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  PhaseSpace ps(inpcrd, CoordinateFileKind::AMBER_INPCRD);
  if (opt.quantize) {
    quantizeCoordinates(&ps);
  }
  const StaticExclusionMask se(&ag);
  const NeckGeneralizedBornTable ngb_tab;
  RecordWriter rw(out);
  putTopology(&rw, ag);
  putExclusionMask(&rw, se);
  putNeckTable(&rw, ngb_tab);
  PhaseSpaceWriter psw = ps.data();
  putCoordinates(&rw, "coords", psw);
  const ValenceKit<double> vk = ag.getDoublePrecisionValenceKit();
  const NonbondedKit<double> nbk = ag.getDoublePrecisionNonbondedKit();
  const ImplicitSolventKit<double> isk = ag.getDoublePrecisionImplicitSolventKit();
  const NeckGeneralizedBornKit<double> ngbk = ngb_tab.dpData();
  ScoreCard sc(1, 1, 32);

  // Per-term FP64 energies (double sums) and forces
  std::vector<double> esum;
  zeroForces(psw);
  esum.push_back(evaluateBondTerms(vk, psw, &sc, EvaluateForce::YES, 0));
  putForces(&rw, "frc_bond", psw);
  zeroForces(psw);
  esum.push_back(evaluateAngleTerms(vk, psw, &sc, EvaluateForce::YES, 0));
  putForces(&rw, "frc_angle", psw);
  zeroForces(psw);
  const double2 dihe = evaluateDihedralTerms(vk, psw, &sc, EvaluateForce::YES, 0);
  esum.push_back(dihe.x);
  esum.push_back(dihe.y);
  putForces(&rw, "frc_dihedral", psw);
  zeroForces(psw);
  const double2 a14 = evaluateAttenuated14Terms(vk, nbk, psw, &sc, EvaluateForce::YES,
                                                EvaluateForce::YES, 0);
  putForces(&rw, "frc_14", psw);
  zeroForces(psw);
  const double2 nb = evaluateNonbondedEnergy(nbk, se.data(), psw, &sc, EvaluateForce::YES,
                                             EvaluateForce::YES, 0);
  putForces(&rw, "frc_nonbonded", psw);
  esum.push_back(nb.y);
  esum.push_back(a14.y);
  esum.push_back(nb.x);
  esum.push_back(a14.x);
  zeroForces(psw);
  std::vector<double> egb(psw.natom), psi(psw.natom), sdeijda(psw.natom);
  const double gb = evaluateGeneralizedBornEnergy<double, double, double>(
                      nbk, se.data(), isk, ngbk, psw.xcrd, psw.ycrd, psw.zcrd, psw.xfrc,
                      psw.yfrc, psw.zfrc, egb.data(), psi.data(), sdeijda.data(), &sc,
                      EvaluateForce::YES, 0);
  esum.push_back(gb);
  putForces(&rw, "frc_gb", psw);
  rw.d("gb_psi", psi);
  rw.d("gb_radii", egb);
  rw.d("gb_sumdeijda", sdeijda);
  rw.d("energy_terms", esum);
  putScoreCard(&rw, "energy_terms_fixed", sc);

  // CHARMM terms: FP64 energy of each kind (Urey-Bradley, CHARMM improper, CMAP), the
  // ScoreCard's fixed-point sums of the same, and the forces of each kind
  {
    std::vector<double> ce, cf;
    ScoreCard sc_ch(1, 1, 32);
    zeroForces(psw);
    ce.push_back(evaluateUreyBradleyTerms(vk, psw, &sc_ch, EvaluateForce::YES, 0));
    putForces(&rw, "frc_ubrd", psw);
    zeroForces(psw);
    ce.push_back(evaluateCharmmImproperTerms(vk, psw, &sc_ch, EvaluateForce::YES, 0));
    putForces(&rw, "frc_cimp", psw);
    zeroForces(psw);
    ce.push_back(evaluateCmapTerms(vk, psw, &sc_ch, EvaluateForce::YES, 0));
    putForces(&rw, "frc_cmap", psw);
    rw.d("charmm_terms", ce);
    for (StateVariable sv : {StateVariable::UREY_BRADLEY, StateVariable::CHARMM_IMPROPER,
                             StateVariable::CMAP}) {
      cf.push_back(sc_ch.reportInstantaneousStates(sv, 0));
    }
    rw.d("charmm_terms_fixed", cf);
  }

  // The complete evaluation through the MM driver STORMM uses for single points
  zeroForces(psw);
  ScoreCard sc_all(1, 1, 26);
  const RestraintApparatus ra(&ag);
  evalRestrainedMMGB(&ps, &sc_all, ag, ngb_tab, se, ra, EvaluateForce::YES, 0);
  putForces(&rw, "frc_total", psw);
  putScoreCard(&rw, "energy_terms_mm", sc_all);
  {
    std::vector<double> cm;
    for (StateVariable sv : {StateVariable::UREY_BRADLEY, StateVariable::CHARMM_IMPROPER,
                             StateVariable::CMAP}) {
      cm.push_back(sc_all.reportInstantaneousStates(sv, 0));
    }
    rw.d("charmm_terms_mm", cm);
  }
  if (opt.clash_r0 >= 0.0 || opt.clash_ratio >= 0.0) {
    const double r0 = (opt.clash_r0 >= 0.0) ? opt.clash_r0 : 0.0;
    const double ratio = (opt.clash_ratio >= 0.0) ? opt.clash_ratio : 0.0;
    zeroForces(psw);
    ScoreCard sc_clash(1, 1, 26);
    evalRestrainedMMGB(&ps, &sc_clash, ag, ngb_tab, se, ra, EvaluateForce::YES, 0, 0, r0, ratio);
    putForces(&rw, "clash_frc_total", psw);
    putScoreCard(&rw, "clash_energy_terms", sc_clash);
    rw.scalar("clash_r0", r0);
    rw.scalar("clash_ratio", ratio);
  }
  return 0;
}

MinimizeControls minimizeControls(const Options &opt) {
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
  mincon.setInitialStep(opt.dx0);
  mincon.setDiagnosticPrintFrequency(1);
  return mincon;
}

int runMinimize(const std::string &prmtop, const std::string &inpcrd, const std::string &out,
                const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  PhaseSpace ps(inpcrd, CoordinateFileKind::AMBER_INPCRD);
  if (opt.quantize) {
    quantizeCoordinates(&ps);
  }
  const StaticExclusionMask se(&ag);
  const NeckGeneralizedBornTable ngb_tab;
  const RestraintApparatus ra(&ag);
  const MinimizeControls mincon = minimizeControls(opt);
  ScoreCard sc = minimize(&ps, ag, ngb_tab, ra, se, mincon);
  RecordWriter rw(out);
  std::vector<double> etot;
  for (StateVariable sv : kTerms) {
    const std::vector<double> h = sc.reportHistory(sv, 0);
    if (etot.empty()) {
      etot.assign(h.size(), 0.0);
    }
    for (size_t k = 0; k < h.size() && k < etot.size(); k++) {
      etot[k] += h[k];
    }
  }
  rw.d("min_potential_history", etot);
  rw.scalar("min_final_potential", sc.reportPotentialEnergy(0));
  putCoordinates(&rw, "min_final_coords", ps.data());
  std::vector<double> efinal;
  for (StateVariable sv : kTerms) {
    efinal.push_back(sc.reportInstantaneousStates(sv, 0));
  }
  rw.d("min_final_terms", efinal);
  return 0;
}

int runTime(const std::string &list_file, double seconds, const Options &opt) {
  std::ifstream lst(list_file);
  std::vector<AtomGraph> ags;
  std::vector<PhaseSpace> pss;
  std::string top, crd;
  while (lst >> top >> crd) {
    ags.push_back(loadTopology(top, opt));
    pss.emplace_back(crd, CoordinateFileKind::AMBER_INPCRD);
  }
  if (ags.empty()) {
    std::fprintf(stderr, "no systems listed in %s\n", list_file.c_str());
    return 2;
  }
  std::vector<StaticExclusionMask> ses;
  std::vector<RestraintApparatus> ras;
  for (size_t i = 0; i < ags.size(); i++) {
    ses.emplace_back(&ags[i]);
    ras.emplace_back(&ags[i]);
  }
  const NeckGeneralizedBornTable ngb_tab;
  const auto t0 = std::chrono::steady_clock::now();
  double elapsed = 0.0;
  long long count = 0;
  size_t idx = 0;
  double checksum = 0.0;
  while (elapsed < seconds) {
    if (opt.minimize_cycles > 0) {
      Options o2 = opt;
      o2.maxcyc = opt.minimize_cycles;
      PhaseSpace ps_copy = pss[idx];
      const MinimizeControls mincon = minimizeControls(o2);
      ScoreCard sc = minimize(&ps_copy, ags[idx], ngb_tab, ras[idx], ses[idx], mincon);
      checksum += sc.reportInstantaneousStates(StateVariable::POTENTIAL_ENERGY, 0);
    }
    else {
      ScoreCard sc(1, 1, 26);
      pss[idx].initializeForces();
      evalRestrainedMMGB(&pss[idx], &sc, ags[idx], ngb_tab, ses[idx], ras[idx],
                         EvaluateForce::YES, 0);
      checksum += sc.reportInstantaneousStates(StateVariable::POTENTIAL_ENERGY, 0);
    }
    count++;
    idx = (idx + 1) % ags.size();
    elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  std::printf("%s=%lld seconds=%.6f systems=%zu checksum=%.6f\n",
              (opt.minimize_cycles > 0) ? "minimizations" : "evals", count, elapsed, ags.size(),
              checksum);
  return 0;
}

// STORMM's MdlMol parse of every compound of an SD / MOL file: per compound its atom and bond
// counts, coordinates, atomic numbers, formal charges and element symbols, the bonds as
// STORMM writes them back (writeMdl, V2000 bond lines: 1-based atoms and the bond type), and
// the data items' names and lines
int runSdf(const std::string &path, const std::string &out) {
  const std::vector<structure::MdlMol> mols = structure::readStructureDataFile(path);
  RecordWriter rw(out);
  rw.iscalar("compounds", static_cast<int>(mols.size()));
  for (size_t m = 0; m < mols.size(); m++) {
    const std::string p = "c" + std::to_string(m) + "_";
    const structure::MdlMol &mol = mols[m];
    const int n = mol.getAtomCount();
    rw.iscalar(p + "natom", n);
    std::vector<double> xyz;
    for (int i = 0; i < n; i++) {
      const double3 c = mol.getCoordinates(i);
      xyz.push_back(c.x);
      xyz.push_back(c.y);
      xyz.push_back(c.z);
    }
    rw.d(p + "xyz", xyz);
    rw.i(p + "znum", mol.getAtomicNumbers());
    rw.i(p + "charge", mol.getFormalCharges());
    std::vector<int> sym;
    for (int i = 0; i < n; i++) {
      const char4 c = mol.getAtomSymbol(i);
      sym.push_back(c.x);
      sym.push_back(c.y);
      sym.push_back(c.z);
      sym.push_back(c.w);
    }
    rw.i(p + "symbols", sym);
    // bond block of STORMM's own V2000 rendering: the fourth line after the atoms onward
    const std::string text = mol.writeMdl(structure::MdlMolVersion::V2000);
    std::vector<std::string> lines;
    size_t a = 0;
    while (a < text.size()) {
      const size_t b = text.find('\n', a);
      lines.push_back(text.substr(a, (b == std::string::npos ? text.size() : b) - a));
      a = (b == std::string::npos) ? text.size() : b + 1;
    }
    std::vector<int> bonds;
    for (int k = 0; k < mol.getBondCount(); k++) {
      const std::string &ln = lines[4 + n + k];
      bonds.push_back(std::atoi(ln.substr(0, 3).c_str()) - 1);
      bonds.push_back(std::atoi(ln.substr(3, 3).c_str()) - 1);
      bonds.push_back(std::atoi(ln.substr(6, 3).c_str()));
    }
    rw.i(p + "bonds", bonds);
    rw.iscalar(p + "items", mol.getDataItemCount());
    for (int k = 0; k < mol.getDataItemCount(); k++) {
      const std::string q = p + "item" + std::to_string(k) + "_";
      const std::string name = mol.getDataItemName(k);
      std::vector<int> chars(name.begin(), name.end());
      rw.i(q + "name", chars);
      std::string content;
      for (const std::string &line : mol.getDataItemContent(k)) {
        if (!content.empty()) content += '\n';
        content += line;
      }
      std::vector<int> cchars(content.begin(), content.end());
      rw.i(q + "content", cchars);
    }
  }
  return 0;
}

// STORMM's clash verdict (detectClash with its default clash distance and ratio) for each
// coordinate file of <list-file> (one inpcrd per line) under one topology, and the
// mass-weighted aligned RMSD (RMSDMethod::ALIGN_MASS) of each against the first
int runGeometry(const std::string &prmtop, const std::string &list_file, const std::string &out,
                const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  const StaticExclusionMask se(&ag);
  std::ifstream lst(list_file);
  std::string crd;
  std::vector<CoordinateFrame> frames;
  while (lst >> crd) {
    frames.emplace_back(crd, CoordinateFileKind::AMBER_INPCRD);
  }
  std::vector<int> clash;
  std::vector<double> rms;
  for (const CoordinateFrame &cf : frames) {
    clash.push_back(structure::detectClash(cf, ag, se, default_minimize_clash_r0,
                                           default_minimize_clash_ratio) ? 1 : 0);
    rms.push_back(structure::rmsd(frames[0], cf, ag, structure::RMSDMethod::ALIGN_MASS));
  }
  RecordWriter rw(out);
  rw.i("clash", clash);
  rw.d("rmsd_to_first", rms);
  return 0;
}

// An Amber input-coordinate file as STORMM writes it (PhaseSpace::exportToFile,
// CoordinateFileKind::AMBER_INPCRD) after reading the coordinates of another one
int runWriteCrd(const std::string &in, const std::string &out) {
  PhaseSpace ps(in, CoordinateFileKind::AMBER_INPCRD);
  ps.exportToFile(out, 0.0, TrajectoryKind::POSITIONS, CoordinateFileKind::AMBER_INPCRD,
                  PrintSituation::OVERWRITE);
  return 0;
}

int runNbwu(const std::string &list_file, const std::string &out, const Options &opt,
             int init_task) {
  std::ifstream lst(list_file);
  std::vector<std::string> tops;
  std::vector<int> counts;
  std::string top;
  int count = 0;
  while (lst >> top >> count) {
    tops.push_back(top);
    counts.push_back(count);
  }
  std::vector<AtomGraph> ags;
  ags.reserve(tops.size());
  for (const std::string &t : tops) {
    ags.push_back(loadTopology(t, opt));
  }
  std::vector<AtomGraph*> ag_ptrs;
  std::vector<int> index;
  for (size_t k = 0; k < ags.size(); k++) {
    ag_ptrs.push_back(&ags[k]);
    for (int c = 0; c < counts[k]; c++) {
      index.push_back(static_cast<int>(k));
    }
  }
  synthesis::AtomGraphSynthesis poly_ag(ag_ptrs, index);
  const synthesis::StaticExclusionMaskSynthesis poly_se(ag_ptrs, index);
  poly_ag.loadNonbondedWorkUnits(poly_se, static_cast<synthesis::InitializationTask>(init_task),
                                 0, card::GpuDetails());
  const synthesis::SyNonbondedKit<double, double2> nbk = poly_ag.getDoublePrecisionNonbondedKit();
  const synthesis::SeMaskSynthesisReader ser = poly_se.data();
  RecordWriter rw(out);
  rw.i("index", index);
  rw.i("se_atom_counts", ser.atom_counts, ser.nsys);
  rw.i("se_atom_offsets", ser.atom_offsets, ser.nsys);
  rw.i("se_supertile_map_bounds", ser.supertile_map_bounds, ser.nsys + 1);
  rw.i("se_supertile_map_idx", ser.supertile_map_idx, ser.supertile_map_bounds[ser.nsys]);
  rw.i("se_tile_map_idx", ser.tile_map_idx, 256 * static_cast<size_t>(ser.nsupertile));
  rw.u("se_mask_data", ser.mask_data, 32 * static_cast<size_t>(ser.ntile));
  const size_t abs_len = 64;
  rw.i("nbwu_abstracts", nbk.nbwu_abstracts, abs_len * nbk.nnbwu);
  int insr_end = 0;
  for (int w = 0; w < nbk.nnbwu; w++) {
    insr_end = std::max(insr_end, nbk.nbwu_abstracts[abs_len * w + 27]);
  }
  const int insr_count = ((insr_end + 31) / 32) * 32;
  std::vector<uint> insr(2 * static_cast<size_t>(insr_count));
  for (int k = 0; k < insr_count; k++) {
    insr[2 * k] = nbk.nbwu_insr[k].x;
    insr[2 * k + 1] = nbk.nbwu_insr[k].y;
  }
  rw.u("nbwu_insr", insr.data(), insr.size());
  std::printf("work units %d, instructions %d\n", nbk.nnbwu, insr_count);
  return 0;
}

// Surface area of every molecule of one structure, by STORMM's CPU code
int runSasa(const std::string &prmtop, const std::string &inpcrd, int npts,
            const std::string &out, const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  PhaseSpace ps(inpcrd, CoordinateFileKind::AMBER_INPCRD);
  if (opt.quantize) {
    quantizeCoordinates(&ps);
  }
  const std::vector<int> mols = incrementingSeries<int>(0, ag.getMoleculeCount());
  const std::vector<double3> pts = surfaceDistribution<double, double3>(npts);
  std::vector<double> flat;
  for (const double3 &p : pts) {
    flat.push_back(p.x);
    flat.push_back(p.y);
    flat.push_back(p.z);
  }
  const double area = surfaceArea(&ps, &ag, mols, npts, default_sasa_probe_radius, 1.0,
                                  EvaluateForce::NO, SasaReference::LENNARD_JONES_SIGMA,
                                  PrecisionModel::DOUBLE);
  const double energy = surfaceArea(&ps, &ag, mols, npts, default_sasa_probe_radius,
                                    default_sasa_energy, EvaluateForce::NO,
                                    SasaReference::LENNARD_JONES_SIGMA, PrecisionModel::DOUBLE);
  RecordWriter rw(out);
  PhaseSpaceWriter psw = ps.data();
  putCoordinates(&rw, "coords", psw);
  rw.d("sphere_points", flat);
  rw.scalar("sasa_area", area);
  rw.scalar("sasa_energy", energy);
  std::printf("points %zu, area %.10f, energy %.10f\n", pts.size(), area, energy);
  return 0;
}

// Time-dependent restraints on one structure, evaluated by STORMM's CPU code at several steps
int runRestraintRamp(const std::string &prmtop, const std::string &inpcrd,
                     const std::string &list, const std::string &steps, const std::string &out,
                     const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  PhaseSpace ps(inpcrd, CoordinateFileKind::AMBER_INPCRD);
  if (opt.quantize) {
    quantizeCoordinates(&ps);
  }
  std::ifstream in(list);
  std::vector<BoundedRestraint> rs;
  int kind, a[4], s0, s1;
  double v[18];
  while (in >> kind >> a[0] >> a[1] >> a[2] >> a[3] >> s0 >> s1) {
    for (int m = 0; m < 18; m++) {
      in >> v[m];
    }
    const double3 t0 = { v[6], v[7], v[8] };
    const double3 t1 = { v[15], v[16], v[17] };
    switch (kind) {
    case 1:
      rs.emplace_back(a[0], &ag, s0, s1, v[0], v[1], v[2], v[3], v[4], v[5], v[9], v[10], v[11],
                      v[12], v[13], v[14], t0, t1);
      break;
    case 2:
      rs.emplace_back(a[0], a[1], &ag, s0, s1, v[0], v[1], v[2], v[3], v[4], v[5], v[9], v[10],
                      v[11], v[12], v[13], v[14]);
      break;
    case 3:
      rs.emplace_back(a[0], a[1], a[2], &ag, s0, s1, v[0], v[1], v[2], v[3], v[4], v[5], v[9],
                      v[10], v[11], v[12], v[13], v[14]);
      break;
    default:
      rs.emplace_back(a[0], a[1], a[2], a[3], &ag, s0, s1, v[0], v[1], v[2], v[3], v[4], v[5],
                      v[9], v[10], v[11], v[12], v[13], v[14]);
      break;
    }
  }
  RecordWriter rw(out);
  PhaseSpaceWriter psw = ps.data();
  putCoordinates(&rw, "coords", psw);
  std::stringstream ss(steps);
  std::string tok;
  while (std::getline(ss, tok, ',')) {
    const int step = std::atoi(tok.c_str());
    std::vector<double> each;
    for (const BoundedRestraint &r : rs) {
      const RestraintApparatus one(std::vector<BoundedRestraint>(1, r), &ag);
      ScoreCard sc1(1, 1, 32);
      each.push_back(evaluateRestraints(one, &ps, &sc1, EvaluateForce::NO, 0, step));
    }
    const RestraintApparatus ra(rs, &ag);
    ScoreCard sc(1, 1, 32);
    zeroForces(psw);
    const double total = evaluateRestraints(ra, &ps, &sc, EvaluateForce::YES, 0, step);
    putForces(&rw, "frc_restraint_" + tok, psw);
    rw.d("restraint_energies_" + tok, each);
    rw.scalar("restraint_total_" + tok, total);
    std::printf("step %d: restraints %zu, energy %.10f\n", step, rs.size(), total);
  }
  return 0;
}

// Constant restraints of several kinds on one structure, evaluated by STORMM's CPU code
int runRestraint(const std::string &prmtop, const std::string &inpcrd, const std::string &list,
                 const std::string &out, const Options &opt) {
  AtomGraph ag = loadTopology(prmtop, opt);
  PhaseSpace ps(inpcrd, CoordinateFileKind::AMBER_INPCRD);
  if (opt.quantize) {
    quantizeCoordinates(&ps);
  }
  std::ifstream in(list);
  std::vector<BoundedRestraint> rs;
  int kind, a[4];
  double k2, k3, r1, r2, r3, r4, x, y, z;
  while (in >> kind >> a[0] >> a[1] >> a[2] >> a[3] >> k2 >> k3 >> r1 >> r2 >> r3 >> r4 >> x >>
         y >> z) {
    switch (kind) {
    case 1:
      rs.emplace_back(a[0], &ag, k2, k3, r1, r2, r3, r4, double3{x, y, z});
      break;
    case 2:
      rs.emplace_back(a[0], a[1], &ag, k2, k3, r1, r2, r3, r4);
      break;
    case 3:
      rs.emplace_back(a[0], a[1], a[2], &ag, k2, k3, r1, r2, r3, r4);
      break;
    default:
      rs.emplace_back(a[0], a[1], a[2], a[3], &ag, k2, k3, r1, r2, r3, r4);
      break;
    }
  }
  RecordWriter rw(out);
  PhaseSpaceWriter psw = ps.data();
  std::vector<double> each;
  for (const BoundedRestraint &r : rs) {
    const RestraintApparatus one(std::vector<BoundedRestraint>(1, r), &ag);
    ScoreCard sc1(1, 1, 32);
    each.push_back(evaluateRestraints(one, &ps, &sc1, EvaluateForce::NO, 0, 0));
  }
  const RestraintApparatus ra(rs, &ag);
  ScoreCard sc(1, 1, 32);
  zeroForces(psw);
  const double total = evaluateRestraints(ra, &ps, &sc, EvaluateForce::YES, 0, 0);
  putCoordinates(&rw, "coords", psw);
  putForces(&rw, "frc_restraint", psw);
  rw.d("restraint_energies", each);
  rw.scalar("restraint_total", total);
  std::printf("restraints %zu, energy %.10f\n", rs.size(), total);
  return 0;
}

// Valence work units of one topology, with the inputs they are built from
int runVwu(const std::string &prmtop, const std::string &out, const Options &opt, int atoms) {
  const AtomGraph ag = loadTopology(prmtop, opt);
  const ValenceKit<double> vk = ag.getDoublePrecisionValenceKit();
  const NonbondedKit<double> nbk = ag.getDoublePrecisionNonbondedKit();
  const ChemicalDetailsKit cdk = ag.getChemicalDetailsKit();
  if (atoms <= 0) {
    energy::ValenceKernelSize kw;
    atoms = synthesis::calculateValenceWorkUnitSize(std::vector<int>(1, ag.getAtomCount()), 148,
                                                    &kw).x;
  }
  const RestraintApparatus ra(&ag);
  const std::vector<synthesis::ValenceWorkUnit> units =
      synthesis::buildValenceWorkUnits(&ag, &ra, {atoms, atoms});
  RecordWriter rw(out);
  rw.iscalar("natom", ag.getAtomCount());
  rw.iscalar("atom_limit", atoms);
  rw.i("z_numbers", cdk.z_numbers, cdk.natom);
  rw.i("nb12_bounds", nbk.nb12_bounds, nbk.natom + 1);
  rw.i("nb12x", nbk.nb12x, nbk.nb12_bounds[nbk.natom]);
  // the decision buildValenceWorkUnits makes for a unit seeded on each atom
  const int water_natom = ag.getWaterResidueSize();
  const std::string water_name = ag.getWaterResidueName();
  std::vector<int> solvent(cdk.natom);
  for (int a = 0; a < cdk.natom; a++) {
    const int m = cdk.mol_home[a];
    const int mn = cdk.mol_limits[m + 1] - cdk.mol_limits[m];
    const char4 rn = cdk.res_names[ag.getResidueIndex(a)];
    const std::string rns = {rn.x, rn.y, rn.z, rn.w};
    solvent[a] = (mn == 1) ||
                 (mn == water_natom && rns.substr(0, water_name.size()) == water_name &&
                  rns.find_first_not_of(' ', water_name.size()) == std::string::npos);
  }
  rw.i("solvent", solvent);
  rw.i("counts_ub_cimp_cmap", std::vector<int>{vk.nubrd, vk.ncimp, vk.ncmap});
  rw.u("bond_relevance", vk.bond_relevance, (vk.nbond + 31) / 32);
  rw.u("angl_relevance", vk.angl_relevance, (vk.nangl + 31) / 32);
  {
    const ConstraintKit<double> cnk = ag.getDoublePrecisionConstraintKit();
    const VirtualSiteKit<double> vsk = ag.getDoublePrecisionVirtualSiteKit();
    rw.i("counts_settle_cgroup_vsite", std::vector<int>{cnk.nsettle, cnk.ngroup, vsk.nsite});
    rw.i("settle_ox", cnk.settle_ox_atoms, cnk.nsettle);
    rw.i("settle_h1", cnk.settle_h1_atoms, cnk.nsettle);
    rw.i("settle_h2", cnk.settle_h2_atoms, cnk.nsettle);
    rw.i("settle_param", cnk.settle_param_idx, cnk.nsettle);
    rw.i("group_bounds", cnk.group_bounds, cnk.ngroup + 1);
    rw.i("group_list", cnk.group_list, cnk.group_bounds[cnk.ngroup]);
    rw.i("group_param", cnk.group_param_idx, cnk.ngroup);
    rw.i("group_param_bounds", cnk.group_param_bounds, cnk.ncnst_param + 1);
  }
  rw.i("bond_i", vk.bond_i_atoms, vk.nbond);
  rw.i("bond_j", vk.bond_j_atoms, vk.nbond);
  rw.i("bond_param", vk.bond_param_idx, vk.nbond);
  rw.i("angl_i", vk.angl_i_atoms, vk.nangl);
  rw.i("angl_j", vk.angl_j_atoms, vk.nangl);
  rw.i("angl_k", vk.angl_k_atoms, vk.nangl);
  rw.i("angl_param", vk.angl_param_idx, vk.nangl);
  rw.i("dihe_i", vk.dihe_i_atoms, vk.ndihe);
  rw.i("dihe_j", vk.dihe_j_atoms, vk.ndihe);
  rw.i("dihe_k", vk.dihe_k_atoms, vk.ndihe);
  rw.i("dihe_l", vk.dihe_l_atoms, vk.ndihe);
  rw.i("dihe_param", vk.dihe_param_idx, vk.ndihe);
  rw.i("dihe14_param", vk.dihe14_param_idx, vk.ndihe);
  std::vector<int> kind(vk.ndihe);
  for (int k = 0; k < vk.ndihe; k++) {
    kind[k] = static_cast<int>(vk.dihe_modifiers[k].w);
  }
  rw.i("dihe_kind", kind);
  rw.i("infr14_i", vk.infr14_i_atoms, vk.ninfr14);
  rw.i("infr14_l", vk.infr14_l_atoms, vk.ninfr14);
  rw.i("infr14_param", vk.infr14_param_idx, vk.ninfr14);
  // per unit, concatenated: bounds arrays give each unit's range
  std::vector<int> imp, imp_b{0}, upd_flags, upd_b{0}, manip, manip_b{0}, tasks;
  std::vector<int> lists[4], list_b[4], cbnd_list, cbnd_b{0}, cdhe_list, cdhe_b{0};
  std::vector<uint> acc[6], cbnd_insr, angl_insr, cdhe_insr, infr_insr, sett_insr, cnst_insr;
  std::vector<int> moved, sett_b{0}, cnst_b{0};
  std::vector<int> acc_b[6];
  for (int t = 0; t < 6; t++) acc_b[t].push_back(0);
  for (int t = 0; t < 4; t++) list_b[t].push_back(0);
  const synthesis::VwuTask simple[4] = {synthesis::VwuTask::BOND, synthesis::VwuTask::ANGL,
                                        synthesis::VwuTask::DIHE, synthesis::VwuTask::INFR14};
  const synthesis::VwuTask acc_tasks[6] = {synthesis::VwuTask::BOND, synthesis::VwuTask::ANGL,
                                           synthesis::VwuTask::DIHE, synthesis::VwuTask::CBND,
                                           synthesis::VwuTask::CDHE, synthesis::VwuTask::INFR14};
  for (const synthesis::ValenceWorkUnit &u : units) {
    const std::vector<int> il = u.getAtomImportList();
    imp.insert(imp.end(), il.begin(), il.end());
    imp_b.push_back(imp.size());
    const std::vector<uint> uf = u.getAtomUpdateFlags();
    for (uint w : uf) upd_flags.push_back(static_cast<int>(w));
    upd_b.push_back(upd_flags.size());
    for (const uint2 m : u.getAtomManipulationMasks()) {
      manip.push_back(static_cast<int>(m.x));
      manip.push_back(static_cast<int>(m.y));
    }
    manip_b.push_back(manip.size());
    const std::vector<int> tc = u.getTaskCounts();
    tasks.insert(tasks.end(), tc.begin(), tc.end());
    for (int t = 0; t < 4; t++) {
      const std::vector<int> &l = u.getSimpleTaskList(simple[t]);
      lists[t].insert(lists[t].end(), l.begin(), l.end());
      list_b[t].push_back(lists[t].size());
    }
    const std::vector<int> &cb = u.getCompositeBondTaskList();
    cbnd_list.insert(cbnd_list.end(), cb.begin(), cb.end());
    cbnd_b.push_back(cbnd_list.size());
    for (const int2 c : u.getCompositeDihedralTaskList()) {
      cdhe_list.push_back(c.x);
      cdhe_list.push_back(c.y);
    }
    cdhe_b.push_back(cdhe_list.size());
    for (int t = 0; t < 6; t++) {
      const std::vector<uint> &a = u.getAccumulationFlags(acc_tasks[t]);
      acc[t].insert(acc[t].end(), a.begin(), a.end());
      acc_b[t].push_back(acc[t].size());
    }
    for (const uint2 v : u.getCompositeBondInstructions()) {
      cbnd_insr.push_back(v.x);
      cbnd_insr.push_back(v.y);
    }
    for (const uint2 v : u.getAngleInstructions()) {
      angl_insr.push_back(v.x);
      angl_insr.push_back(v.y);
    }
    for (const uint3 v : u.getCompositeDihedralInstructions()) {
      cdhe_insr.push_back(v.x);
      cdhe_insr.push_back(v.y);
      cdhe_insr.push_back(v.z);
    }
    for (const uint v : u.getInferred14Instructions()) {
      infr_insr.push_back(v);
    }
    for (const uint2 v : u.getSettleGroupInstructions()) {
      sett_insr.push_back(v.x);
      sett_insr.push_back(v.y);
    }
    sett_b.push_back(sett_insr.size());
    for (const uint2 v : u.getConstraintGroupInstructions()) {
      cnst_insr.push_back(v.x);
      cnst_insr.push_back(v.y);
    }
    cnst_b.push_back(cnst_insr.size());
    moved.push_back(u.getMovedAtomCount());
  }
  rw.iscalar("nunit", units.size());
  rw.i("imports", imp);
  rw.i("imports_bounds", imp_b);
  rw.i("update_flags", upd_flags);
  rw.i("update_flags_bounds", upd_b);
  rw.i("manip", manip);
  rw.i("manip_bounds", manip_b);
  rw.i("task_counts", tasks);
  const char* lnames[4] = {"bond", "angl", "dihe", "infr14"};
  for (int t = 0; t < 4; t++) {
    rw.i(std::string(lnames[t]) + "_terms", lists[t]);
    rw.i(std::string(lnames[t]) + "_terms_bounds", list_b[t]);
  }
  rw.i("cbnd_terms", cbnd_list);
  rw.i("cbnd_terms_bounds", cbnd_b);
  rw.i("cdhe_terms", cdhe_list);
  rw.i("cdhe_terms_bounds", cdhe_b);
  const char* anames[6] = {"bond", "angl", "dihe", "cbnd", "cdhe", "infr14"};
  for (int t = 0; t < 6; t++) {
    rw.u(std::string("acc_") + anames[t], acc[t].data(), acc[t].size());
    rw.i(std::string("acc_") + anames[t] + "_bounds", acc_b[t]);
  }
  rw.u("cbnd_insr", cbnd_insr.data(), cbnd_insr.size());
  rw.u("angl_insr", angl_insr.data(), angl_insr.size());
  rw.u("cdhe_insr", cdhe_insr.data(), cdhe_insr.size());
  rw.u("infr14_insr", infr_insr.data(), infr_insr.size());
  rw.u("settle_insr", sett_insr.data(), sett_insr.size());
  rw.i("settle_insr_bounds", sett_b);
  rw.u("cgroup_insr", cnst_insr.data(), cnst_insr.size());
  rw.i("cgroup_insr_bounds", cnst_b);
  rw.i("moved_counts", moved);
  std::printf("atoms %d, limit %d, units %zu\n", ag.getAtomCount(), atoms, units.size());
  return 0;
}

// calculateValenceWorkUnitSize over syntheses given as lines of atom counts
int runVwuSize(const std::string &counts_file, int sm_count, const std::string &out) {
  std::ifstream in(counts_file);
  std::string line;
  std::vector<int> sizes, widths;
  while (std::getline(in, line)) {
    std::vector<int> counts;
    size_t p = 0;
    while (p < line.size()) {
      size_t q = line.find(' ', p);
      if (q == std::string::npos) q = line.size();
      if (q > p) counts.push_back(std::atoi(line.substr(p, q - p).c_str()));
      p = q + 1;
    }
    if (counts.empty()) continue;
    if (sm_count > 0) {
      energy::ValenceKernelSize kw;
      const int2 sz = synthesis::calculateValenceWorkUnitSize(counts, sm_count, &kw);
      sizes.push_back(sz.x);
      widths.push_back(static_cast<int>(kw));
    }
    else {
      const int2 sz = synthesis::calculateValenceWorkUnitSize(counts);
      sizes.push_back(sz.x);
      widths.push_back(-1);
    }
  }
  RecordWriter rw(out);
  rw.i("sizes", sizes);
  rw.i("widths", widths);
  return 0;
}

} // namespace

int main(int argc, char* argv[]) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s eval|minimize|time ...\n", argv[0]);
    return 2;
  }
  const std::string mode(argv[1]);
  std::vector<std::string> pos;
  Options opt;
  int init_task = 3;
  int vwu_atoms = 0;
  for (int i = 2; i < argc; i++) {
    const std::string a(argv[i]);
    auto next = [&]() -> double {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", a.c_str());
        std::exit(2);
      }
      return std::atof(argv[++i]);
    };
    if (a == "--igb") opt.igb = static_cast<int>(next());
    else if (a == "--diel") opt.diel = next();
    else if (a == "--salt") opt.salt = next();
    else if (a == "--qtol") opt.qtol = next();
    else if (a == "--qdisc") opt.qdisc = next();
    else if (a == "--scee") opt.scee = next();
    else if (a == "--scnb") opt.scnb = next();
    else if (a == "--maxcyc") opt.maxcyc = static_cast<int>(next());
    else if (a == "--ncyc") opt.ncyc = static_cast<int>(next());
    else if (a == "--dx0") opt.dx0 = next();
    else if (a == "--minimize") opt.minimize_cycles = static_cast<int>(next());
    else if (a == "--cdcyc") opt.cdcyc = static_cast<int>(next());
    else if (a == "--clash-r0") opt.clash_r0 = next();
    else if (a == "--clash-ratio") opt.clash_ratio = next();
    else if (a == "--quantize") opt.quantize = true;
    else if (a == "--init-task") init_task = static_cast<int>(next());
    else if (a == "--vwu-atoms") vwu_atoms = static_cast<int>(next());
    else pos.push_back(a);
  }
  if (mode == "eval" && pos.size() == 3) {
    return runEval(pos[0], pos[1], pos[2], opt);
  }
  if (mode == "minimize" && pos.size() == 3) {
    return runMinimize(pos[0], pos[1], pos[2], opt);
  }
  if (mode == "nbwu" && pos.size() == 2) {
    return runNbwu(pos[0], pos[1], opt, init_task);
  }
  if (mode == "sdf" && pos.size() == 2) {
    return runSdf(pos[0], pos[1]);
  }
  if (mode == "geometry" && pos.size() == 3) {
    return runGeometry(pos[0], pos[1], pos[2], opt);
  }
  if (mode == "restraint" && pos.size() == 4) {
    return runRestraint(pos[0], pos[1], pos[2], pos[3], opt);
  }
  if (mode == "sasa" && pos.size() == 4) {
    return runSasa(pos[0], pos[1], std::atoi(pos[2].c_str()), pos[3], opt);
  }
  if (mode == "restraintramp" && pos.size() == 5) {
    return runRestraintRamp(pos[0], pos[1], pos[2], pos[3], pos[4], opt);
  }
  if (mode == "vwu" && pos.size() == 2) {
    return runVwu(pos[0], pos[1], opt, vwu_atoms);
  }
  if (mode == "vwusize" && pos.size() == 3) {
    return runVwuSize(pos[0], std::atoi(pos[1].c_str()), pos[2]);
  }
  if (mode == "writecrd" && pos.size() == 2) {
    return runWriteCrd(pos[0], pos[1]);
  }
  if (mode == "time" && pos.size() == 2) {
    return runTime(pos[0], std::atof(pos[1].c_str()), opt);
  }
  std::fprintf(stderr, "bad arguments for mode %s\n", mode.c_str());
  return 2;
}
