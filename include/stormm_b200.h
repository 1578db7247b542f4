/*
 * stormm_b200: C ABI of the B200-native batched implicit-solvent molecular-mechanics path.
 *
 * This is the drop-in boundary beneath STORMM's C++ API for one hot path: batched, non-periodic
 * Coulomb + Lennard-Jones with exclusions and scaled 1-4 terms, the Generalized Born passes
 * (Born radii, GB energy and dE/dR, radii chain-rule force), valence terms (bonds, angles,
 * dihedrals), and the line-minimization driver built on them.  Every entry point takes plain
 * pointers, sizes and a CUDA stream; none takes a C++ or torch type.  Entry points return
 * SB_OK (0) or a negative SB_ERR_* code; sb_last_error() describes the last failure on the
 * calling thread.
 *
 * Reference interfaces replaced (paths inside the STORMM source tree):
 *   sb_synthesis_create      AtomGraphSynthesis + PhaseSpaceSynthesis + StaticExclusionMaskSynthesis
 *                            + ImplicitSolventWorkspace + ScoreCard construction
 *                            (Synthesis/atomgraph_synthesis.h:84-110, phasespace_synthesis.h:348-376,
 *                            static_mask_synthesis.h:54, implicit_solvent_workspace.h:83,
 *                            Potential/scorecard.h:110; setImplicitSolventModel
 *                            atomgraph_synthesis.h:455-473)
 *   sb_initialize            PhaseSpaceSynthesis::initializeForces, ImplicitSolventWorkspace::initialize,
 *                            ScoreCard::initialize (phasespace_synthesis.h, kPsyInitializeForces
 *                            hpc_phasespace_synthesis.cu:243; hpc_implicit_solvent_workspace.cu:21;
 *                            hpc_scorecard.cu:17)
 *   sb_launch_nonbonded      launchNonbonded (Potential/hpc_nonbonded_potential.h:142-157)
 *   sb_launch_valence        launchValence (Potential/hpc_valence_potential.h:167-230)
 *   sb_evaluate              launchNonbonded followed by launchValence, fused into one pass
 *   sb_evaluate_clash        the same with the clash_min_dist / clash_ratio arguments
 *   sb_minimize              launchMinimization (MolecularMechanics/hpc_minimization.h:122-152)
 */
#ifndef STORMM_B200_H
#define STORMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status codes                                                                                */
/* ------------------------------------------------------------------------------------------ */
#define SB_OK 0
#define SB_ERR_ARGUMENT -1     /* an argument is out of range or inconsistent */
#define SB_ERR_CUDA -2         /* a CUDA runtime call failed */
#define SB_ERR_DEVICE -3       /* no usable sm_100 device */
#define SB_ERR_UNSUPPORTED -4  /* a feature outside this path (e.g. neck GB) was requested */
#define SB_ERR_KERNEL -5       /* a kernel reported an error through its status word */

/* ------------------------------------------------------------------------------------------ */
/* Enumerations (values follow STORMM's)                                                       */
/* ------------------------------------------------------------------------------------------ */
/* Generalized Born model, as Amber's igb keyword: 0 none, 1 HCT, 2 OBC-I, 5 OBC-II */
#define SB_GB_NONE 0
#define SB_GB_HCT 1
#define SB_GB_OBC 2
#define SB_GB_OBC2 5
#define SB_GB_NECK 7           /* Mongan's neck GB (GBn) */
#define SB_GB_NECK2 8          /* neck GB model II (GBn2): element-specific alpha / beta / gamma */

/* Energy slots per system, STORMM's StateVariable order (Potential/energy_enumerators.h:36-50) */
#define SB_BOND 0
#define SB_ANGLE 1
#define SB_PROPER_DIHEDRAL 2
#define SB_IMPROPER_DIHEDRAL 3
#define SB_UREY_BRADLEY 4
#define SB_CHARMM_IMPROPER 5
#define SB_CMAP 6
#define SB_VDW 7
#define SB_VDW_ONE_FOUR 8
#define SB_ELECTROSTATIC 9
#define SB_ELEC_ONE_FOUR 10
#define SB_GENERALIZED_BORN 11
#define SB_RESTRAINT 12
#define SB_NRG_STRIDE 16        /* energy slots per system in sb_get_energies output */

/* Terms to evaluate (bit mask) */
#define SB_TERM_VALENCE 1
#define SB_TERM_NONBONDED 2     /* Coulomb + Lennard-Jones */
#define SB_TERM_GB 4
#define SB_TERM_ALL 7

/* What sb_initialize clears (bit mask) */
#define SB_INIT_FORCES 1
#define SB_INIT_ENERGIES 2
#define SB_INIT_GB_WORKSPACE 4

/* ------------------------------------------------------------------------------------------ */
/* Inputs                                                                                      */
/* ------------------------------------------------------------------------------------------ */
/* One molecule's topology (host memory, 0-based atom indices).  The fields are what STORMM's
 * AtomGraph provides through its NonbondedKit, ValenceKit and ImplicitSolventKit
 * (Topology/atomgraph_abstracts.h:88-377). */
typedef struct {
  int natom;
  const double* charge;        /* natom, elementary charges */
  const int* lj_idx;           /* natom, Lennard-Jones type of each atom */
  int n_lj_types;
  const double* lja;           /* n_lj_types^2, A coefficients (kcal/mol A^12) */
  const double* ljb;           /* n_lj_types^2, B coefficients (kcal/mol A^6) */
  const double* lja14;         /* n_lj_types^2, 1-4 A coefficients (NULL: same as lja) */
  const double* ljb14;         /* n_lj_types^2, 1-4 B coefficients (NULL: same as ljb) */
  const int* excl_bounds;      /* natom + 1, CSR bounds of each atom's excluded partners */
  const int* excl_list;        /* 1-2, 1-3 and 1-4 partners of each atom (either order) */
  const double* pb_radii;      /* natom, intrinsic GB radii (A) */
  const double* gb_screen;     /* natom, GB screening factors */
  const double* gb_alpha;      /* natom, OBC alpha (NULL: model defaults) */
  const double* gb_beta;       /* natom */
  const double* gb_gamma;      /* natom */
  int nbond;
  const int* bond_atoms;       /* 2 * nbond */
  const double* bond_keq;      /* kcal/mol A^2 */
  const double* bond_leq;      /* A */
  int nangl;
  const int* angl_atoms;       /* 3 * nangl */
  const double* angl_keq;      /* kcal/mol rad^2 */
  const double* angl_theta0;   /* rad */
  int ndihe;
  const int* dihe_atoms;       /* 4 * ndihe */
  const double* dihe_amp;      /* kcal/mol */
  const double* dihe_freq;     /* periodicity */
  const double* dihe_phase;    /* rad */
  const double* dihe_scee;     /* 1-4 electrostatic attenuation, 0 when the term carries no 1-4 */
  const double* dihe_scnb;     /* 1-4 Lennard-Jones attenuation */
  const int* dihe_improper;    /* nonzero: energy is reported as improper (NULL: all proper) */
  /* CHARMM terms (all zero / NULL for Amber force fields), evaluated in FP64 by a kernel of
   * their own after the fused pass (Potential/valence_potential.tpp:659-1300) */
  int nubrd;                   /* Urey-Bradley 1-3 harmonic stretches */
  const int* ubrd_atoms;       /* 2 * nubrd (atoms i, k) */
  const double* ubrd_keq;      /* kcal/mol A^2 */
  const double* ubrd_leq;      /* A */
  int ncimp;                   /* CHARMM harmonic impropers: k (theta - phase)^2 */
  const int* cimp_atoms;       /* 4 * ncimp */
  const double* cimp_keq;      /* kcal/mol rad^2 */
  const double* cimp_phase;    /* rad */
  int ncmap;                   /* CMAP terms: a bicubic spline surface over two dihedrals */
  const int* cmap_atoms;       /* 5 * ncmap: phi is atoms 0-3, psi atoms 1-4 */
  const int* cmap_surface;     /* ncmap surface indices */
  int ncmap_surf;
  const int* cmap_dims;        /* grid points per side of each surface */
  const double* cmap_values;   /* surfaces back to back, kcal/mol: the value at phi index j and
                                  psi index k is at j + k * dim, grid point j at -180 + j * 360 /
                                  dim degrees */
} sb_topology;

typedef struct {
  int igb;                     /* SB_GB_* */
  double dielectric;           /* solvent dielectric (STORMM default 80) */
  double saltcon;              /* salt concentration, mol/L */
  double coulomb_constant;     /* kcal A / mol e^2 (STORMM/Amber 332.05221729) */
  int gpos_bits;               /* fixed-point bits of coordinates (32) */
  int frc_bits;                /* fixed-point bits of forces (23) */
  int nrg_bits;                /* fixed-point bits of energies (26) */
  int max_atoms_per_unit;      /* work-unit packing limit, 0: tuned default */
  int max_tiles_per_unit;      /* work-unit packing limit, 0: tuned default */
  int threads_per_block;       /* 0: tuned default */
  int device;                  /* CUDA device ordinal */
  int tiled_above_atoms;       /* molecules with more atoms are evaluated tile by tile from global
                                  memory, spread over the whole GPU (0: 2048, the on-chip limit;
                                  32-2048); the graph minimizer minimizes them, the persistent
                                  one refuses them */
  int precision;               /* SB_PRECISION_SINGLE (default): FP32 arithmetic with fixed-point
                                  accumulation; SB_PRECISION_DOUBLE: FP64 arithmetic from double
                                  parameters (STORMM's PrecisionModel::DOUBLE), every molecule tile
                                  by tile; minimized by the graph minimizer with an FP64 direction */
  /* Neck GB (igb 7, 8): STORMM's NeckGeneralizedBornTable, neck_table_size^2 maximum
   * separations and values indexed [j_index * size + i_index], with the per-atom index
   * round(20 (r_pb - 1)) (radii must lie in [1, 2] A); read by sb_synthesis_create */
  const double* neck_max_separation;
  const double* neck_max_value;
  int neck_table_size;
  double neck_cut;             /* neck cutoff, A (STORMM's default 6.8) */
} sb_options;

#define SB_PRECISION_SINGLE 0
#define SB_PRECISION_DOUBLE 1

/* Fill *opt with STORMM's defaults (OBC-II, dielectric 80, no salt, 32/23/26 fixed-point bits) */
void sb_default_options(sb_options* opt);

typedef struct sb_synthesis sb_synthesis;

/* Build a synthesis of nsys systems.  System k uses topology tops[topology_index[k]].  All device
 * memory is allocated here and released by sb_synthesis_destroy. */
int sb_synthesis_create(const sb_topology* tops, int ntop, const int* topology_index, int nsys,
                        const sb_options* opt, sb_synthesis** out);
int sb_synthesis_destroy(sb_synthesis* syn);

int sb_system_count(const sb_synthesis* syn);
/* Atom count of one system and the offset of its first atom in the padded device arrays */
int sb_system_atoms(const sb_synthesis* syn, int system, int* natom, int* offset);
/* Total padded atom count (every system starts on a multiple of 32) */
int sb_padded_atom_count(const sb_synthesis* syn);

/* ------------------------------------------------------------------------------------------ */
/* Host <-> device transfers.  xyz arrays hold all systems back to back without padding,       */
/* 3 doubles per atom.  Each call is one copy plus a conversion kernel on the stream.          */
/* ------------------------------------------------------------------------------------------ */
/* Asynchronous: with a pinned host buffer the caller must keep it unchanged until the stream
 * reaches this point.  Non-finite or out-of-range coordinates leave those atoms unchanged and
 * set bit 2 of the status word (sb_check_status). */
int sb_set_coordinates(sb_synthesis* syn, const double* xyz, void* stream);
/* The getters synchronize the stream before returning. */
int sb_get_coordinates(sb_synthesis* syn, double* xyz, void* stream);
int sb_get_forces(sb_synthesis* syn, double* xyz, void* stream);
/* energies: nsys * SB_NRG_STRIDE doubles, kcal/mol, STORMM's slot order */
int sb_get_energies(sb_synthesis* syn, double* energies, void* stream);
/* No counterpart in the reference (PhaseSpaceSynthesis::download and ScoreCard::download wait):
 * the forces and energies of sb_get_forces / sb_get_energies enqueued on the stream without
 * waiting, into page-locked host buffers (refused otherwise), complete once the stream reaches
 * this point; either may be NULL.  A serving loop with two syntheses on two streams overlaps
 * one batch's transfers with the other's evaluation. */
int sb_download_results_async(sb_synthesis* syn, double* forces, double* energies, void* stream);
/* GB intermediates per atom (unpadded): psi (A^-1), effective radii (A), sum of dE/dR
 * after the chain-rule prefactor, as STORMM's ImplicitSolventWorkspace holds them */
int sb_get_gb_workspace(sb_synthesis* syn, double* psi, double* radii, double* sumdeijda,
                        void* stream);
/* Raw fixed-point arrays (padded layout) for bit-exact inspection: int64 x, y, z + int32 overflow */
int sb_get_forces_fixed(sb_synthesis* syn, int64_t* xyz_primary, int32_t* xyz_overflow,
                        void* stream);
int sb_get_energies_fixed(sb_synthesis* syn, int64_t* energies, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Evaluation                                                                                  */
/* ------------------------------------------------------------------------------------------ */
int sb_initialize(sb_synthesis* syn, int what, void* stream);
/* All requested terms for every system in one fused pass.  Forces and energies accumulate
 * into the synthesis' arrays (clear them with sb_initialize first). */
int sb_evaluate(sb_synthesis* syn, int terms, int eval_force, int eval_energy, void* stream);
/* Systems [first, first + count) only: the per-system drop-in launch sequence */
int sb_evaluate_range(sb_synthesis* syn, int first, int count, int terms, int eval_force,
                      int eval_energy, void* stream);
/* STORMM's two launchers, each alone */
int sb_launch_nonbonded(sb_synthesis* syn, int eval_force, int eval_energy, void* stream);
int sb_launch_valence(sb_synthesis* syn, int eval_force, int eval_energy, void* stream);
/* sb_evaluate with clash mitigation, the clash_min_dist / clash_ratio arguments of
 * launchNonbonded and launchValence (hpc_nonbonded_potential.h:142-157,
 * hpc_valence_potential.h:167-230): Coulomb and Lennard-Jones pairs, 1-4 pairs included, take
 * a quadratic Coulomb core below clash_distance (A) and a quartic Lennard-Jones core below
 * clash_ratio times the pair's sigma = (A/B)^(1/6) (Potential/soft_core_potentials.tpp).  Both
 * zero is the plain evaluation; GB terms are never softened. */
int sb_evaluate_clash(sb_synthesis* syn, int terms, int eval_force, int eval_energy,
                      double clash_distance, double clash_ratio, void* stream);

/* Number of work units the batched launches use, and the launch shape chosen: threads is the
 * block size of the evaluation launch of packed units (512 when that launch holds fewer units
 * than one wave of 256-thread blocks, unless sb_autotune found 256 faster or threads_per_block
 * fixes it) */
int sb_launch_info(const sb_synthesis* syn, int* work_units, int* blocks, int* threads);

/* ------------------------------------------------------------------------------------------ */
/* Line minimization                                                                           */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's MinimizeControls for the GPU minimizer (Namelists/nml_minimize.h:21-30,
 * MolecularMechanics/hpc_minimization.h:122-152) */
typedef struct {
  int total_cycles;            /* maxcyc: line-minimization cycles (STORMM default 200) */
  int sd_cycles;               /* ncyc: steepest-descent cycles before conjugate gradient (50) */
  int clash_cycles;            /* cdcyc: leading cycles evaluated with softened cores (STORMM's
                                  namelist default is 25; 0 here) */
  double initial_step;         /* dx0: first move length, A (0.01) */
  double convergence_rms;      /* a system stops once its RMS force (kcal/mol/A, over 3N
                                  components) is at or below this; 0: run every cycle, as
                                  STORMM's GPU minimizer does */
  int record_history;          /* nonzero: keep each system's energy at the start of every cycle
                                  and the final energy (total_cycles + 1 values per system) */
  int kernel;                  /* SB_MIN_GRAPH (default) or SB_MIN_PERSISTENT */
  double clash_distance;       /* clash_r0: softened-core distance in cycle 0 (0.2 A) */
  double clash_ratio;          /* clash_vdw_ratio: softened-core sigma ratio in cycle 0 (0.5);
                                  cycle c < clash_cycles uses both scaled by
                                  (clash_cycles - c) / clash_cycles, counted per system, and the
                                  final energy is undamped (hpc_minimization.cu:266-279) */
} sb_minimize_controls;

/* How a minimization runs.  Both follow the same algorithm; their FP32 evaluations are separate
 * compiled codes, so their trajectories agree to rounding, not bit for bit.
 *   SB_MIN_GRAPH       each cycle is one CUDA graph, captured once per synthesis: the batched
 *                      evaluation kernel (force + energy, then three energy-only evaluations)
 *                      with a per-system line-search kernel after each
 *   SB_MIN_PERSISTENT  one persistent kernel runs every cycle of a work unit on chip */
#define SB_MIN_GRAPH 0
#define SB_MIN_PERSISTENT 1

void sb_default_minimize_controls(sb_minimize_controls* ctl);

/* Minimize every system from its current coordinates: steepest descent for sd_cycles, then
 * conjugate gradient, each cycle a force evaluation and a four-point line search with a cubic
 * fit, as launchMinimization (hpc_minimization.h:122-152).  Coordinates move in place; on return
 * (stream order) the energies hold each system's final energy terms.  The whole minimization is
 * one kernel launch per molecule size class. */
int sb_minimize(sb_synthesis* syn, const sb_minimize_controls* ctl, void* stream);
/* Systems [first, first + count) with one launch per system: the per-system drop-in sequence */
int sb_minimize_range(sb_synthesis* syn, int first, int count, const sb_minimize_controls* ctl,
                      void* stream);
/* The same minimization in steps: sb_minimize_begin resets every system's minimizer state
 * (move length dx0, no previous force or direction, zero cycles) without moving anything;
 * each sb_minimize_advance runs up to `cycles` more cycles of every system that has neither
 * converged nor reached total_cycles, and with final_energy nonzero re-evaluates the energies
 * at the coordinates reached.  Begin + one advance of total_cycles equals sb_minimize, and the
 * trajectory does not depend on how the cycles are split between advances. */
int sb_minimize_begin(sb_synthesis* syn, const sb_minimize_controls* ctl, void* stream);
int sb_minimize_advance(sb_synthesis* syn, int cycles, int final_energy, void* stream);

/* The line-search steps one at a time, for a caller that runs its own evaluations in between, as
 * STORMM's launchMinimization does with its kernels (hpc_minimization.cu:432-560).  Both need a
 * minimization begun by sb_minimize_begin and act on every system of the synthesis.
 *
 * sb_conjugate_gradient replaces launchConjugateGradient (Math/hpc_reduction.h:55-63, kernels
 * Math/conjugate_gradient.cui:8-140): from the forces and energies of a force + energy evaluation
 * at the line start it records the energy in the history, takes gg, dgg and the RMS force per
 * system (FP64, over 32-atom chunks in a fixed order), stops a system that met the RMS target
 * or used up total_cycles, and sets the search direction to the forces plus gamma = dgg / gg
 * times the previous direction (gamma = 0 for the first sd_cycles cycles).
 *
 * sb_line_advance replaces launchLineAdvance (MolecularMechanics/hpc_minimization.h:63-70,
 * line_movement.cui:88-336) for move_number 0-3, after an energy evaluation at the current
 * coordinates (move 0: the line-start evaluation itself): move 0 records the line-start energy
 * and moves each active system along its normalized direction by its move length; moves 1 and 2
 * read the trial energy and move on by factors of 1.04 / 0.8 and x1.03 / x0.85; move 3 reads
 * the fourth energy, places the system at the minimum of the cubic through the four points,
 * updates its move length and ends its cycle.
 *
 * Per cycle: clear forces and energies, force + energy evaluation, sb_conjugate_gradient,
 * sb_line_advance(0), then three times: clear energies, energy evaluation, sb_line_advance(1, 2,
 * 3).  With the evaluations of sb_evaluate this is, bit for bit, the cycle of sb_minimize with the
 * graph kernel and no clash-damped cycles. */
int sb_conjugate_gradient(sb_synthesis* syn, void* stream);
int sb_line_advance(sb_synthesis* syn, int move_number, void* stream);

/* Energy history of the last minimization that recorded one: nsys * (total_cycles + 1) doubles,
 * system-major.  Entry c is the energy at the start of cycle c; the entry after a system's last
 * cycle is its final energy (later entries stay 0 for a system that converged early). */
int sb_get_minimize_history(sb_synthesis* syn, double* history, void* stream);
/* Per system: cycles completed, whether the RMS force target was met, latest RMS force.  Any
 * output may be NULL. */
int sb_get_minimize_progress(sb_synthesis* syn, int* cycles_done, int* converged,
                             double* rms_force, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Request server: continuous batching of minimization requests                                */
/* ------------------------------------------------------------------------------------------ */
/* No single counterpart in the reference: it serves conformer-minimization requests the way
 * apps/Conf/src/conformer.cpp:118-172 drives launchMinimization, but as a stream.  A worker
 * thread admits queued requests into batches while an HBM budget allows, keeps each batch's
 * topology, coordinates and minimizer state resident on the device, runs its minimization in
 * launches of cycles_per_launch cycles on a stream of its own (batches overlap on the GPU),
 * retires every molecule that converged or reached total_cycles after each launch, and
 * backfills: new batches start while older ones are still running, and when all but
 * migrate_fraction of a minimization batch have retired while minimizations wait, its remaining
 * molecules move with
 * their minimizer state into a new batch beside the waiting requests and the old batch's memory
 * is released (persistent FP32 minimizer).  A molecule's result does not depend on the batch it
 * ran in, nor on a move.
 *
 * Errors: submit checks the topology on the host (the checks the synthesis applies) and refuses
 * a bad request with its error code; the server's controls are checked when it is created.  A
 * batch that still fails to build is split and its requests are retried one per batch, so only
 * the request that cannot be built fails; a request that fails is returned by poll with its
 * error code in status.  Only a lost CUDA context stops the worker: the batches in flight are
 * returned failed, and submit and drain then report the error (poll still hands out the
 * results that were ready). */
#define SB_TIMEOUT 1            /* sb_server_drain: work still in flight when time ran out */

typedef struct {
  sb_options options;                /* GB model, fixed-point bits, device */
  sb_minimize_controls controls;     /* per request: cycle cap, convergence target, ... */
  double hbm_budget_bytes;           /* device memory for molecules in flight (estimated) */
  int max_batch_molecules;           /* most molecules admitted into one batch */
  int max_batches;                   /* batches in flight at once, one CUDA stream each */
  int cycles_per_launch;             /* minimization cycles per launch of a batch */
  double migrate_fraction;           /* move a minimization batch's remaining molecules into a
                                        new batch once this fraction of it or less remains and
                                        minimizations wait, in [0, 1); 0: never (default 0.25) */
} sb_server_options;

#define SB_REQUEST_MINIMIZE 0          /* run the minimization, return the final coordinates */
#define SB_REQUEST_EVALUATE 1          /* one force + energy evaluation, return the forces */

typedef struct {
  long long request_id;
  int natom;
  int kind;                          /* SB_REQUEST_* */
  int cycles;                        /* line-minimization cycles run */
  int converged;                     /* nonzero: the RMS force met controls.convergence_rms */
  int status;                        /* SB_OK, or the error code that failed the request (no
                                        coordinates or forces are returned for it) */
  double rms_force;                  /* kcal/mol/A at the start of the last cycle (minimization),
                                        at the given coordinates (evaluation) */
  double energy;                     /* total potential energy at the final coordinates */
  double energies[SB_NRG_STRIDE];    /* the terms, StateVariable order */
  double submit_time;                /* seconds since the server started */
  double admit_time;
  double finish_time;
} sb_served_result;

typedef struct {
  long long submitted;
  long long admitted;
  long long completed;                /* results returned, the failed ones included */
  long long failed;                   /* requests returned with an error status */
  long long migrated;                 /* molecule moves out of an emptying batch into a new one */
  int pending;                       /* queued, not yet admitted */
  int in_flight;                     /* admitted molecules still minimizing */
  int batches;
  double bytes_in_flight;
} sb_server_stats;

typedef struct sb_server sb_server;

/* Defaults: OBC-II, controls as sb_default_minimize_controls with total_cycles 2000,
 * convergence_rms 0.01 and the persistent kernel (lower latency for small batches), 2 GB budget,
 * 512 molecules per batch, 16 batches, 50 cycles a launch */
void sb_default_server_options(sb_server_options* opt);
int sb_server_create(const sb_server_options* opt, sb_server** out);
/* Queue one molecule for minimization (topology and coordinates are copied); thread-safe */
int sb_server_submit(sb_server* srv, const sb_topology* top, const double* xyz,
                     long long* request_id);
/* Queue one molecule for a force + energy evaluation at the given coordinates.  Evaluation
 * requests are batched with each other (a batch holds one kind of request), admitted under the
 * same HBM budget and overlap on the device with the minimization batches in flight. */
int sb_server_submit_evaluation(sb_server* srv, const sb_topology* top, const double* xyz,
                                long long* request_id);
/* Completed requests, oldest first: up to max_results, each with its natom * 3 doubles packed
 * into xyz (in result order) while xyz_capacity doubles last: the final coordinates of a
 * minimization, the forces (kcal/mol/A) of an evaluation.  xyz may be NULL to take results
 * without them.  *count receives the number returned. */
int sb_server_poll(sb_server* srv, sb_served_result* results, int max_results, double* xyz,
                   long long xyz_capacity, int* count);
/* Wait until nothing is queued or in flight and every batch's device memory is released: SB_OK,
 * or SB_TIMEOUT after timeout_seconds */
int sb_server_drain(sb_server* srv, double timeout_seconds);
int sb_server_get_stats(sb_server* srv, sb_server_stats* stats);
/* Stops the worker after the launches in flight and releases everything */
int sb_server_destroy(sb_server* srv);

/* ------------------------------------------------------------------------------------------ */
/* STORMM's exclusion-mask tables                                                              */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's StaticExclusionMask of one topology (Potential/static_exclusionmask.cpp:20-260, the
 * per-system part of StaticExclusionMaskSynthesis, Synthesis/static_mask_synthesis.h:54), built
 * on the host in STORMM's layout from the topology's exclusion lists: 256-atom supertiles and
 * 16 x 16 tiles, supertile_map_idx (stride^2 ints), tile_map_idx (256 ints per stored
 * supertile) and mask_data (32 words per stored tile).  Host only, no device needed.  Each
 * n_* is the capacity of its array on input (ignored when the array is NULL) and the size
 * needed on output: call once with NULL arrays to size them. */
int sb_static_exclusion_mask(const sb_topology* top, int* supertile_stride_count,
                             int* supertile_map_idx, long long* n_supertile_map,
                             int* tile_map_idx, long long* n_tile_map, uint32_t* mask_data,
                             long long* n_mask_data);

/* STORMM's StaticExclusionMaskSynthesis tables for nsys systems (system k uses
 * tops[topology_index[k]]), built as Synthesis/static_mask_synthesis.cpp:84-200 combines the
 * per-topology tables: supertile_map_bounds (nsys + 1 ints, caller-sized), supertile_map_idx,
 * tile_map_idx and mask_data with the sizing protocol of sb_static_exclusion_mask.  Host only. */
int sb_static_exclusion_mask_synthesis(const sb_topology* tops, int ntop,
                                       const int* topology_index, int nsys,
                                       int* supertile_map_bounds, int* supertile_map_idx,
                                       long long* n_supertile_map, int* tile_map_idx,
                                       long long* n_tile_map, uint32_t* mask_data,
                                       long long* n_mask_data);

/* STORMM's nonbonded work units for the same synthesis, as buildNonbondedWorkUnits and
 * AtomGraphSynthesis::loadNonbondedWorkUnits lay them out (Synthesis/nonbonded_workunit.cpp:
 * 454-755, nonbonded_workunit.tpp:8-150, ag_synthesis_mechanics.cpp:2668-2730): 64-int
 * abstracts per unit (import count, up to 20 import starts, packed import sizes, instruction
 * range, import systems, initialization mask, refresh start and code) and the tile
 * instructions, two words (x: import slots, y: mask offset in the synthesis tables) per tile,
 * each unit's list padded with zeros to a multiple of 32.  init_task is STORMM's
 * InitializationTask (0 GENERAL_DYNAMICS ... 3 GB_MINIMIZATION ... 6 NONE); refresh work is
 * assigned as with no GPU given.  The kernels of this library use their own work units; these
 * tables are for callers that keep STORMM's.  Syntheses large enough for STORMM's 256-tile
 * units return SB_ERR_UNSUPPORTED.  Sizing as sb_static_exclusion_mask. */
int sb_nonbonded_work_units(const sb_topology* tops, int ntop, const int* topology_index,
                            int nsys, int init_task, int random_cache_depth, int* abstracts,
                            long long* n_abstracts, uint32_t* instructions,
                            long long* n_instructions);

/* ------------------------------------------------------------------------------------------ */
/* Restraints                                                                                  */
/* ------------------------------------------------------------------------------------------ */
/* STORMM's flat-bottom restraints (Restraints/bounded_restraint.h, evaluated as
 * Potential/valence_potential.tpp:1558-2050 and Restraints/restraint_util.tpp:9-77): for the
 * restrained value d (distance from the target point, distance between two atoms, angle, or
 * dihedral angle in radians), the energy is k2 (d - r2)^2 between r1 and r2, zero between r2 and
 * r3, k3 (d - r3)^2 between r3 and r4, and continues linearly below r1 and above r4.  A dihedral
 * is taken within pi of (r2 + r3) / 2.  Energies go to slot SB_RESTRAINT.
 *
 * Time dependence (computeRestraintMixture): at step s, a restraint is absent while
 * s < init_step; with init_step == final_step it then holds its initial values (the final ones
 * are ignored, so a zero-filled tail is a constant restraint from step 0); otherwise the
 * stiffnesses, bounds and target are (1 - w) initial + w final with
 * w = (s - init_step) / (final_step - init_step) up to final_step, and the final values after.
 * The step is the synthesis's restraint step (sb_set_restraint_step, 0 by default) for
 * evaluations, and each system's completed cycle count inside the graph minimizer (the cycle's
 * four evaluations at its index, the final evaluation at the cycles run), as STORMM's
 * minimizer hands its cycle counter to the restraints. */
#define SB_RESTRAINT_POSITION 1
#define SB_RESTRAINT_DISTANCE 2
#define SB_RESTRAINT_ANGLE 3
#define SB_RESTRAINT_DIHEDRAL 4

typedef struct {
  int system;                  /* system of the synthesis */
  int kind;                    /* SB_RESTRAINT_*: the restraint involves that many atoms */
  int atoms[4];                /* atom indices within the system (unused ones ignored) */
  double k2, k3;               /* stiffness of the lower and upper walls (kcal/mol per unit^2) */
  double r1, r2, r3, r4;       /* bounds, ascending (A, or radians for angles and dihedrals) */
  double target[3];            /* positional restraints: the reference point (A) */
  int init_step, final_step;   /* steps at which the restraint engages and is complete */
  double final_k2, final_k3;   /* values at final_step (used when final_step > init_step) */
  double final_r1, final_r2, final_r3, final_r4;
  double final_target[3];
} sb_restraint;

/* Replace the synthesis's restraints (count 0 removes them); evaluated with the valence terms
 * and by the graph minimizer (the persistent minimizer refuses restrained syntheses). */
int sb_set_restraints(sb_synthesis* syn, const sb_restraint* restraints, int count);

/* STORMM's sphere-point surface area of every system (Potential/surface_area.cpp:46-99 and
 * surface_area.tpp:28-173, as apps/Gbsa/src/mmgbsa.cpp:248 calls it: every molecule, radii half
 * the Lennard-Jones sigma of the (type 0, atom type) pair-table entry, double precision) at the
 * synthesis's current coordinates: for each atom, n_points points (sphere_points, 3 doubles each,
 * on the unit sphere) at its radius plus probe_radius; a point counts 4 pi (radius + probe)^2 /
 * n_points unless it lies strictly inside another atom's enlarged sphere in the same or the
 * next-lower cell along each axis of the reference's grid.  out[s] = area * weight (weight 1:
 * A^2; STORMM's default 0.005 kcal/mol per A^2, probe 1.4 A).  Synchronous on the stream. */
int sb_surface_area(sb_synthesis* syn, const double* sphere_points, int n_points,
                    double probe_radius, double weight, double* out, void* stream);

/* The step at which evaluations outside the minimizer take time-dependent restraints
 * (non-negative; SB_ERR_ARGUMENT otherwise). */
int sb_set_restraint_step(sb_synthesis* syn, int step);

/* ------------------------------------------------------------------------------------------ */
/* STORMM's valence work units                                                                 */
/* ------------------------------------------------------------------------------------------ */
/* The valence terms and constraint groups of one topology in STORMM's own order and indexing:
 * the fields of its ValenceKit, ConstraintKit and NonbondedKit (Topology/atomgraph_abstracts.h)
 * that buildValenceWorkUnits reads.  Parameter indices are the topology's.  dihe_kind is
 * STORMM's TorsionKind (0 PROPER, 1 PROPER_NO_14, 2 IMPROPER, 3 IMPROPER_NO_14).  The
 * relevance arrays are STORMM's bit masks (bit k of word k / 32 set: term k is evaluated); NULL
 * marks a term relevant when none of its atoms has atomic number 0 (STORMM's rule without
 * SHAKE / SETTLE).  solvent flags the atoms whose molecule is a single atom or a water (NULL:
 * single-atom molecules, found from the 1-2 lists).  Urey-Bradley, CHARMM improper and CMAP
 * terms, restraints and virtual sites are not represented; atoms of atomic number 0 are
 * refused. */
typedef struct {
  int natom;
  const int* z_numbers;          /* natom atomic numbers (NULL: all nonzero) */
  const int* nb12_bounds;        /* natom + 1, CSR bounds of each atom's 1-2 partners */
  const int* nb12_list;
  const int* solvent;            /* natom flags (NULL: from the 1-2 lists) */
  int nbond;
  const int* bond_i;
  const int* bond_j;
  const int* bond_param;
  const uint32_t* bond_relevance;
  int nangl;
  const int* angl_i;
  const int* angl_j;
  const int* angl_k;
  const int* angl_param;
  const uint32_t* angl_relevance;
  int ndihe;
  const int* dihe_i;
  const int* dihe_j;
  const int* dihe_k;
  const int* dihe_l;
  const int* dihe_param;
  const int* dihe14_param;       /* 1-4 scaling-factor pair of each dihedral */
  const int* dihe_kind;
  int ninfr14;                   /* inferred 1-4 pairs (not carried by a dihedral) */
  const int* infr14_i;
  const int* infr14_l;
  const int* infr14_param;
  int nsettle;                   /* SETTLE groups (rigid waters) */
  const int* settle_ox;
  const int* settle_h1;
  const int* settle_h2;
  const int* settle_param;
  int ngroup;                    /* hub-and-spoke constraint groups, central atom first */
  const int* group_bounds;       /* ngroup + 1 */
  const int* group_list;
  const int* group_param;
  const int* group_param_bounds; /* offsets of each group parameter set's bond lengths */
} sb_valence_topology;

typedef struct sb_valence_units sb_valence_units;

/* STORMM's valence work units of one topology (Synthesis/valence_workunit.cpp:
 * ValenceDelegator, ValenceWorkUnit, buildValenceWorkUnits with a blank RestraintApparatus):
 * units grown from the first unassigned atom through the 1-2 graph up to atom_limit imported
 * atoms (solvent_atom_limit for a unit seeded on a solvent atom), each atom updated by exactly
 * one unit, each term's energy accumulated by the first unit that evaluates it, and the
 * instructions STORMM stores against the topology's own parameter indices.  Limits lie in
 * [32, 512].  Host only.  Release with sb_valence_units_destroy. */
int sb_valence_work_units(const sb_valence_topology* top, int atom_limit, int solvent_atom_limit,
                          sb_valence_units** out);
int sb_valence_units_destroy(sb_valence_units* units);
int sb_valence_unit_count(const sb_valence_units* units, int* count);

#define SB_VWU_TASKS 16          /* STORMM's VwuTask order: BOND ANGL DIHE UBRD CBND CIMP CDHE
                                    CMAP INFR14 RPOSN RBOND RANGL RDIHE VSITE SETTLE CGROUP */

/* One unit, pointers into the set's storage (valid until it is destroyed).  Counts of the term
 * lists and instruction arrays are the task counts; each acc_* mask has (count + 31) / 32 words,
 * bit k set when the unit accumulates the energy of its k-th term of that kind. */
typedef struct {
  int imported_atoms;            /* getImportedAtomCount */
  int moved_atoms;               /* getMovedAtomCount */
  int updated_atoms;             /* getUpdatedAtomCount */
  int task_counts[SB_VWU_TASKS]; /* getTaskCounts */
  int n_manip;                   /* manipulation-mask entries (a multiple of 32) */
  const int* imports;            /* imported atoms, ascending topology indices */
  const uint32_t* manip;         /* n_manip (x, y) pairs: import mask, update mask */
  const uint32_t* update_flags;  /* (imported_atoms + 31) / 32 words: getAtomUpdateFlags */
  const int* bond_terms;         /* topology term indices, ascending */
  const int* angl_terms;
  const int* dihe_terms;
  const int* infr14_terms;
  const int* cbnd_terms;         /* composite bonds: the bonds (no Urey-Bradley terms) */
  const int* cdhe_terms;         /* composite dihedrals: (first, second or -1) pairs */
  const uint32_t* acc_bond;
  const uint32_t* acc_angl;
  const uint32_t* acc_dihe;
  const uint32_t* acc_cbnd;
  const uint32_t* acc_cdhe;
  const uint32_t* acc_infr14;
  const uint32_t* cbnd_insr;     /* 2 words per composite bond */
  const uint32_t* angl_insr;     /* 2 words per angle */
  const uint32_t* cdhe_insr;     /* 3 words per composite dihedral */
  const uint32_t* infr14_insr;   /* 1 word per inferred 1-4 pair */
  const uint32_t* settle_insr;   /* 2 words per SETTLE group */
  const uint32_t* cgroup_insr;   /* 2 words per constraint slot (task_counts[15], padded) */
} sb_valence_unit_view;

int sb_valence_unit(const sb_valence_units* units, int unit, sb_valence_unit_view* view);

/* calculateValenceWorkUnitSize (Synthesis/valence_workunit.cpp, the overload with an SM count)
 * for a synthesis of nsys systems in isolated boundary conditions: the atom limit and STORMM's
 * ValenceKernelSize (0 XL, 1 LG, 2 MD, 3 SM) it picks.  With sm_count <= 0 the overload without
 * one: the size of least padding, kernel width not set. */
int sb_valence_work_unit_size(const int* atom_counts, int nsys, int sm_count, int* atom_limit,
                              int* kernel_width);

/* ------------------------------------------------------------------------------------------ */
/* Amber file intake                                                                           */
/* ------------------------------------------------------------------------------------------ */
/* An Amber topology (prmtop) read from disk: what STORMM's AtomGraph(file_name) reads
 * (Topology/atomgraph.h:83,156, atomgraph_detailers.cpp:677-1120).  Host only, no device
 * needed.  Charges come out in electrons, Lennard-Jones tables expanded to n_types^2, 1-2 / 1-3
 * / 1-4 exclusions from the bond graph, GB radii and screening factors as the file holds them.
 * Refused: nonzero 10-12 hydrogen-bond terms and massless particles (virtual sites,
 * SB_ERR_UNSUPPORTED).  A unit cell is reported in the view and not
 * applied (this path evaluates in isolated boundary conditions); CHARMM Urey-Bradley, improper
 * and CMAP terms are counted in the view but not evaluated. */
typedef struct sb_amber_topology sb_amber_topology;

typedef struct {
  sb_topology topology;             /* ready for sb_synthesis_create; gb_alpha / beta / gamma
                                       are NULL until sb_amber_set_implicit_solvent */
  const int* atomic_numbers;        /* natom (inferred from masses when the file has none) */
  const double* masses;             /* natom, daltons */
  const int* exclusion_bounds[3];   /* natom + 1 each: CSR bounds of the 1-2, 1-3, 1-4 lists */
  const int* exclusion_list[3];     /* partners one, two and three bonds away, ascending */
  const char* radius_set;           /* RADIUS_SET text ("" when absent) */
  const char* title;
  int implicit_solvent;             /* SB_GB_* applied, -1 for none yet */
  int cmap_count;                   /* CHARMM terms present in the file (not evaluated) */
  int urey_bradley_count;
  int charmm_improper_count;
  int unit_cell;                    /* the file's IFBOX (0: none); recorded, not applied */
} sb_amber_view;

int sb_read_amber_topology(const char* prmtop_path, sb_amber_topology** out);
/* Pointers into the topology's own arrays, valid until sb_amber_topology_destroy or the next
 * sb_amber_set_implicit_solvent */
int sb_amber_topology_view(const sb_amber_topology* top, sb_amber_view* view);
/* Radius sets (STORMM's AtomicRadiusSet, Topology/atomgraph_enumerators.h:150-152) */
#define SB_RADII_NONE 0         /* keep the file's radii and screening factors */
#define SB_RADII_BONDI 1
#define SB_RADII_AMBER6 2
#define SB_RADII_MBONDI 3
#define SB_RADII_MBONDI2 4
#define SB_RADII_MBONDI3 5
#define SB_RADII_PARSE 6
/* Per-atom GB parameters of a model as STORMM's AtomGraph::setImplicitSolventModel assigns them
 * (Topology/atomgraph_setters.cpp:672-1060): the radius set's radii and screening factors (the
 * neck models replace file radii outside [1, 2] A by Bondi or mBondi3 radii), then uniform
 * alpha / beta / gamma for HCT, OBC and OBC-II, element screening factors for neck GB, element
 * alpha / beta / gamma and screening factors for neck GB II */
int sb_amber_set_implicit_solvent(sb_amber_topology* top, int igb, int radius_set);
int sb_amber_topology_destroy(sb_amber_topology* top);
/* Coordinates of an Amber ASCII coordinate or restart file (STORMM's PhaseSpace(file_name)):
 * 3 * natom doubles, interlaced x, y, z; the file's atom count must equal natom */
int sb_read_amber_coordinates(const char* inpcrd_path, int natom, double* xyz);
/* Write coordinates (3 * natom doubles, interlaced) as an Amber input-coordinate file, the
 * format STORMM's PhaseSpace::exportToFile writes for CoordinateFileKind::AMBER_INPCRD
 * (Trajectory/write_frame.cpp:54-160): a title line, the atom count as %7d, then six %12.7f
 * values a line; the checkpoint of a minimized structure.  title may be NULL. */
int sb_write_amber_coordinates(const char* inpcrd_path, const char* title, int natom,
                               const double* xyz);

/* ------------------------------------------------------------------------------------------ */
/* MDL MOL / SD files                                                                          */
/* ------------------------------------------------------------------------------------------ */
/* Compounds of an SD file (or one MOL file), V2000 format, as STORMM's MdlMol reads them
 * (MoleculeFormat/mdlmol.cpp:47-324, readStructureDataFile at :1821-1880): coordinates, element
 * symbols and atomic numbers, formal charges (atom-block codes, replaced by "M  CHG"
 * properties), bonds with their MDL types, and the compound's data items.  V3000 compounds are
 * refused (SB_ERR_UNSUPPORTED).  Host only. */
typedef struct sb_sdf sb_sdf;

typedef struct {
  const char* title;
  int natom;
  const double* xyz;                 /* 3 * natom, interlaced, Angstrom */
  const int* atomic_number;          /* natom (0 for a symbol that is no element) */
  const int* formal_charge;          /* natom, electrons */
  const char* symbols;               /* 4 characters per atom, NUL padded */
  int nbond;
  const int* bond_i;                 /* nbond, 0-based */
  const int* bond_j;
  const int* bond_order;             /* MDL bond type: 1-3 single to triple, 4 aromatic, ... */
  int n_items;                       /* data items: "> <name>" and the lines that follow */
  const char* const* item_names;
  const char* const* item_contents;  /* lines joined by '\n' */
} sb_sdf_view;

int sb_read_sdf(const char* path, sb_sdf** out);
int sb_sdf_compound_count(const sb_sdf* sdf, int* count);
/* Pointers into the compound's own arrays, valid until sb_sdf_destroy */
int sb_sdf_compound(const sb_sdf* sdf, int index, sb_sdf_view* view);
int sb_sdf_destroy(sb_sdf* sdf);
/* Write one compound in the V2000 format (coordinates %10.4f as STORMM's MdlMol writes them,
 * charges as "M  CHG" properties, data items, closing "$$$$"), replacing the file or appended
 * to it; the element symbols come from symbols, or from atomic_number when symbols is NULL.
 * Up to 999 atoms and 999 bonds. */
int sb_write_sdf_compound(const char* path, int append, const sb_sdf_view* compound);

/* ------------------------------------------------------------------------------------------ */
/* Autotuning                                                                                  */
/* ------------------------------------------------------------------------------------------ */
#define SB_TUNE_EVALUATE 1
#define SB_TUNE_MINIMIZE 2
/* Times candidate work-unit packings (atom slots and tiles per unit) of the batched evaluation
 * or minimization kernel on this synthesis and keeps the fastest, in place of STORMM's fixed
 * launch tables (Structure/core_kernel_manager.h:83-195).  Results do not depend on the packing.
 * Tuning the evaluation clears forces, energies and the GB workspace; tuning the minimizer
 * leaves coordinates as they were and requires a new sb_minimize_begin before an advance.
 * Outputs may be NULL. */
int sb_autotune(sb_synthesis* syn, int what, int* max_atoms_per_unit, int* max_tiles_per_unit,
                double* best_ms, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Energy export without allocation                                                            */
/* ------------------------------------------------------------------------------------------ */
/* No counterpart in the reference.  Converts nsys * stride int64 energies in device memory
 * (nrg_bits fraction bits, STORMM's ScoreCard format, e.g. a synthesis' or a ScoreCard's device
 * accumulators) to doubles in host memory through a scratch array compiled into the library,
 * allocating nothing.  For callers that must not allocate device memory where they read
 * energies: a loop whose device memory is committed to the work in flight, or a ScoreCard
 * that has no synthesis handle and so no staging buffer.
 * Limit: nsys * stride <= 65,536 values (4,096 systems of 16 slots); larger requests return
 * SB_ERR_ARGUMENT.  The first call on each device (nsys = 0 does only this) looks up the
 * scratch address with that device current: make it before any stream capture begins.  The
 * address is kept with its CUDA context; a call in another context (after cudaDeviceReset, or
 * with a context of the caller's own current) looks it up again, so make a set-up call there
 * too before a capture.
 * Nothing has to be zeroed first.  Calls on one device share the scratch: calls that overlap
 * in time race, so order them.  Synchronizes the stream before returning. */
int sb_energies_to_host_static(const int64_t* d_energies, int nsys, int stride, int nrg_bits,
                               double* energies, void* stream);

/* Read and clear the device status word that bounded device-side waits and checks set */
int sb_check_status(sb_synthesis* syn, int* status);

const char* sb_last_error(void);
const char* sb_version(void);

#ifdef __cplusplus
}
#endif

#endif
