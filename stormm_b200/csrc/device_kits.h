// Device-side views of a synthesis, passed by value to the kernels.  These are internal to the
// library: the C ABI (include/stormm_b200.h) exposes handles, not these layouts.
//
// Layout in HBM (structure of arrays, every system's first atom on a multiple of 32):
//   coordinates  int64 x/y/z, fixed point with gpos_bits fraction bits (STORMM's
//                PhaseSpaceSynthesis, Synthesis/phasespace_synthesis.h:87-197), int32 overflow
//   forces       int64 x/y/z with frc_bits fraction bits + int32 overflow (int95 format,
//                Numerics/split_fixed_precision.h:30-34)
//   energies     int64 per system per StateVariable slot, nrg_bits fraction bits
//   per-atom     charge * sqrt(Coulomb constant), LJ type, offset GB radius rho = r_pb - 0.09,
//   parameters   screened radius s*rho, OBC alpha/beta/gamma, intrinsic radius r_pb
//   valence      16-byte records (uint4) with 16-bit system-local atom indices
//   exclusions   one 32 x 32 bit mask per tile of a system that holds an exclusion
#ifndef STORMM_B200_DEVICE_KITS_H
#define STORMM_B200_DEVICE_KITS_H

#include <cstdint>
#include <vector_types.h>

namespace sb {

constexpr int kTile = 32;                 // atoms per tile edge (one warp lane per atom)
constexpr int kMaxUnitSystems = 32;       // systems per fused work unit
constexpr int kMaxFusedAtoms = 2048;      // largest molecule the fused path holds on chip
constexpr int kNrgStride = 16;            // energy slots per system (STORMM StateVariable order)
constexpr int kUnitMetaFields = 8;        // ints per unit-molecule row of DevSynthesis::unit_meta
constexpr int kPairDerivPerTile = 1024;  // float2 entries per tile of DevSynthesis::pair_deriv
constexpr float kGbRadiiOffset = 0.09f;   // Constants/generalized_born.h:114
constexpr float kGbKscale = 0.73f;        // Constants/generalized_born.h:123
constexpr int kPsiBits = 29;              // fixed-point bits of the in-block psi accumulators
constexpr int kDeijdaBits = 23;           // fixed-point bits of the in-block dE/dR accumulators

// Energy slots (Potential/energy_enumerators.h:36-50)
enum NrgSlot : int {
  kBond = 0, kAngle = 1, kProperDihedral = 2, kImproperDihedral = 3, kVdw = 7, kVdw14 = 8,
  kElec = 9, kElec14 = 10, kGb = 11
};

// Bond record:     x = i | j << 16, y = keq, z = leq (high float), w = leq - z (low float)
// Angle record:    x = i | j << 16, y = k, z = keq, w = cos(theta0)
// Dihedral record: a.x = i | j << 16, a.y = k | l << 16 | improper << 31, a.z = amp, a.w = freq
//                  b.x = cos(phase), b.y = sin(phase), b.z = 1/scee (0: no 1-4), b.w = 1/scnb
// (floats stored as their bit patterns; indices are molecule-local)
struct DevSynthesis {
  int nsys;
  int natom_padded;
  int igb;                       // 0 none, 1 HCT, 2 OBC, 5 OBC-II
  float kappa;                   // Debye-Hueckel kappa from the salt concentration
  float inv_dielectric;
  float frc_scale;               // 2^frc_bits
  float nrg_scale;               // 2^nrg_bits
  double inv_gpos_scale;         // 2^-gpos_bits
  double psi_out_scale;          // 2^24, ImplicitSolventWorkspace's single-precision fp_bits

  // per system
  const int* atom_start;
  const int* atom_count;
  const int* bond_start;         // CSR over systems (nsys + 1)
  const int* angl_start;
  const int* dihe_start;
  const int* lj_start;           // offset of the system's LJ table in ljab
  const int* lj_ntypes;
  const int* tile_start;         // offset of the system's tile-mask index list

  // per atom
  const long long* xcrd;
  const long long* ycrd;
  const long long* zcrd;
  long long* xfrc;
  long long* yfrc;
  long long* zfrc;
  int* xfrc_ovrf;
  int* yfrc_ovrf;
  int* zfrc_ovrf;
  const float* charge;           // q * sqrt(Coulomb constant)
  const int* lj_idx;
  const float* rho;              // r_pb - 0.09
  const float* srho;             // screen * rho
  const float* pb_radii;
  const float* gb_alpha;
  const float* gb_beta;
  const float* gb_gamma;
  // the same GB radius parameters in FP64 (rho, intrinsic radius, alpha, beta; gamma), for the
  // per-atom effective radius and chain-rule factor, whose OBC form cancels for buried atoms
  const double4* gb_radius64;
  const double* gb_gamma64;

  // tables
  const float2* ljab;            // (A, B) per type pair
  const float2* ljab14;
  const uint4* bonds;
  const uint4* angles;
  const uint4* dihe_a;
  const uint4* dihe_b;
  // valence parameters in FP64 for the angle, dihedral and attached 1-4 terms, which evaluate in
  // FP64 from the coordinates' exact hi + lo sums (near-linear angles, near-planar impropers and
  // close 1-4 pairs need more than FP32 deltas and cross products)
  const double4* angl64;         // per angle: k, cos(theta0), sin(theta0), theta0
  const double4* dihe64;         // per dihedral: amplitude, cos(phase), sin(phase), periodicity
  const double4* dihe14_64;      // per dihedral: the attached 1-4 pair's q_i q_l / scee,
                                 // A / scnb, B / scnb, and 1 (all 0: no 1-4 pair)
  const int* tile_mask_idx;      // per system tile, 0: no exclusions, else index into mask_pool
  const unsigned int* mask_pool; // 32 rows per mask: row = i lane, bit = j lane

  // outputs
  unsigned long long* energies;  // nsys * kNrgStride, int64 two's complement
  long long* psi;                // ImplicitSolventWorkspace psi (fixed, 2^24)
  int* psi_ovrf;
  long long* sumdeijda;
  int* sumdeijda_ovrf;
  float* born_radii;             // effective radii of the last evaluation

  // work units, described by unit_desc, molecule tables in unit_meta
  int nunit;
  const int4* unit_desc;         // x = first row in unit_meta, y = system count,
                                 // z = atom slots (sum of padded sizes), w = tile count
  const int* unit_meta;          // kUnitMetaFields ints per unit molecule plus a closing row per
                                 // unit (unit_desc.x is the first row): system, atoms, first
                                 // slot, first tile, LJ table offset, bond / angle / dihedral
                                 // chunk offsets; the closing row holds the totals
  int max_unit_slots;
  // HCT pair derivatives of the work units' tiles, written by GB pass 1 of a force evaluation
  // and read by pass 3: 32 steps x 32 lanes of (i-side, j-side) values per tile, a unit's tiles
  // from the base in its closing unit_meta row
  float2* pair_deriv;

  // neck GB (igb 7, 8): per padded atom its table index, the tables (float), their size (0: not
  // a neck model), and the model's neck scale, cutoff and baseline radius offset
  const int* neck_idx;
  const float* neck_sep;
  const float* neck_val;
  int neck_size;
  float neck_scale;
  float neck_cut;
  float gb_offset;

  // clash damping of a launch (softened Coulomb and Lennard-Jones cores): clash distance (A) and
  // sigma ratio, off when both are 0.  With clash_cycle set (a minimization), system s uses them
  // scaled by (clash_cycles - c) / clash_cycles in its cycle c = clash_cycle[s], and not at all
  // once c >= clash_cycles.
  float clash_distance;
  float clash_ratio;
  int clash_cycles;
  const int* clash_cycle;

  int* status;                   // device status word (0 = fine)
};

// Molecules evaluated tile by tile from global memory (too large for one block's shared memory,
// or routed there by the tiled_above_atoms option): every 32 x 32 tile of every such molecule is
// an independent warp task, so one molecule spreads over the whole GPU.  Pair passes accumulate
// into global integer arrays; per-atom steps run between the passes as separate kernels.
struct DevTiled {
  int nmol;                      // molecules on the tiled path
  int ntiles;                    // their tiles in total
  const int* systems;            // system index of each
  const int* tile_prefix;        // nmol + 1: first tile of each molecule
  const int* atom_prefix;        // nmol + 1: first padded atom of each, counted over these only
  long long* psi_acc;            // per padded atom: psi at 2^kPsiBits
  long long* de_acc;             // per padded atom: dE/dR at 2^kDeijdaBits
  float* radius;                 // per padded atom: effective GB radius
  float* sde;                    // per padded atom: dE/dR after the chain-rule prefactor
};

// Double-precision parameters of the FP64 mode (STORMM's double-precision kits beside the
// single-precision ones), with the same layouts as their FP32 counterparts in DevSynthesis
struct DevPrecise {
  const double* charge;          // per padded atom: charge x sqrt(Coulomb constant)
  const double* rho;             // intrinsic GB radius - 0.09 A
  const double* srho;            // screening factor x rho
  const double* pb_radii;
  const double* alpha;
  const double* beta;
  const double* gamma;
  const double2* ljab;           // per-topology (A, B) tables at DevSynthesis::lj_start offsets
  const double2* ljab14;
  const int2* bond_atoms;        // per bond: molecule-local atoms
  const double2* bond_prm;       // k, r0
  const int4* angl_atoms;        // per angle: i, j, k
  const double2* angl_prm;       // k, theta0
  const int4* dihe_atoms;        // per dihedral: i, j, k, l
  const double4* dihe_prm;       // amplitude, periodicity, phase, 1 for an improper
  const double2* dihe_attn;      // 1 / scee, 1 / scnb of the attached 1-4 pair (0: none)
  double kappa;                  // Debye-Hueckel screening (1/A)
  double inv_dielectric;
  const double* neck_sep;        // neck GB tables (DevSynthesis::neck_size entries squared)
  const double* neck_val;
  double neck_scale;
  double neck_cut;
  double gb_offset;
  double* radius;                // per padded atom: effective GB radius of the evaluation
  double* sde;                   // per padded atom: dE/dR after the chain-rule prefactor
  double clash_distance;         // softened cores, as DevSynthesis' clash fields, in double
  double clash_ratio;
  int clash_cycles;
  const int* clash_cycle;
};

// Line-minimization state (MolecularMechanics/line_minimization.h:15-221 and the conjugate
// gradient substrate, Math/hpc_reduction.h:55-63), per system and per padded atom.  It persists
// between launches, so a minimization can run in several launches of a few cycles each.
struct DevMinimizer {
  long long* xcrd;               // the synthesis' coordinates, moved in place
  long long* ycrd;
  long long* zcrd;
  long long* xprv;               // force of the previous cycle, fixed point with frc_bits
  long long* yprv;
  long long* zprv;
  float* xcg;                    // conjugate-gradient direction (kcal/mol/A, not normalized)
  float* ycg;
  float* zcg;
  double* xcg64;                 // the direction in FP64 (FP64 mode only, else null)
  double* ycg64;
  double* zcg64;
  double* l_move;                // per system: baseline move length (A)
  int* cycle;                    // per system: completed line-minimization cycles
  int* done;                     // per system: nonzero once the RMS force met the target
  double* rms_force;             // per system: RMS force at the start of the latest cycle
  double* history;               // per system: energy at the start of each cycle (may be null)
  int hist_stride;               // history entries per system
  int sd_cycles;                 // steepest-descent cycles before conjugate gradient
  int max_cycles;                // a system stops moving after this many cycles in total
  double drms;                   // RMS force target (kcal/mol/A), 0: none
  int clash_cycles;              // leading cycles with softened cores (0: none)
  float clash_distance;          // their clash distance (A) and sigma ratio in cycle 0
  float clash_ratio;
  int* queue;                    // work-unit counter, zero before each launch
  double* line;                  // per system: kLineFields line-search scalars (graph minimizer)
};

// Line-search scalars per system between the graph minimizer's kernels
enum LineField : int {
  kLineE0 = 0, kLineE1, kLineE2, kLineMv1, kLineMv2, kLineMv3, kLineMfac, kLineSMove,
  kLineInvNorm, kLineAct, kLineFields
};

// CHARMM terms of a synthesis (charmm.cu), atom indices in the padded layout, each term with
// its system; terms are stored system by system
struct DevCharmm {
  const int4* ubrd = nullptr;          // x i, y k, z system
  const double2* ubrd_prm = nullptr;   // keq, leq
  const int4* cimp = nullptr;          // atoms i, j, k, l
  const int* cimp_sys = nullptr;
  const double2* cimp_prm = nullptr;   // keq, phase
  const int4* cmap = nullptr;          // atoms 0-3
  const int4* cmap_b = nullptr;        // x atom 4, y system, z surface
  const int2* cmap_surf = nullptr;     // per surface: first patch (16 doubles each), grid points
  const double* cmap_patch = nullptr;  // 16 bicubic coefficients per grid cell
  const long long* xcrd = nullptr;
  const long long* ycrd = nullptr;
  const long long* zcrd = nullptr;
  long long* xfrc = nullptr;
  long long* yfrc = nullptr;
  long long* zfrc = nullptr;
  unsigned long long* energies = nullptr;
  double inv_gpos_scale = 0.0, frc_scale = 0.0, nrg_scale = 0.0;
  // restraints: atoms in the padded layout (unused ones repeat the first), x kind y system,
  // stiffnesses, bounds r1-r4, positional target
  const int4* rst_atoms = nullptr;
  const int2* rst_meta = nullptr;
  const double2* rst_k = nullptr;
  const double4* rst_r = nullptr;
  const double4* rst_target = nullptr;
  // time dependence: final stiffnesses, bounds and target, the steps at which the restraint
  // engages and is complete, and the step (rst_cycle: per-system cycle counts that replace it)
  const double2* rst_kf = nullptr;
  const double4* rst_rf = nullptr;
  const double4* rst_target_f = nullptr;
  const int2* rst_steps = nullptr;
  int rst_step = 0;
  const int* rst_cycle = nullptr;
};

// Arrays zeroed by one launch of launchClear: 16-byte aligned bases, lengths in 16-byte words
struct ClearList {
  void* ptr[8];
  size_t words[8];
  int count = 0;
};

}  // namespace sb

#endif
