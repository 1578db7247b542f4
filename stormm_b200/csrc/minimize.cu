// Batched line minimization: STORMM's GPU minimizer (MolecularMechanics/hpc_minimization.cu:
// 129-600) restated as one persistent kernel.
//
// STORMM runs each cycle as about thirty launches over the whole synthesis: a force + energy
// evaluation, the conjugate-gradient gather / scatter / rescale (Math/conjugate_gradient.cui),
// then three rounds of line advance + energy-only evaluation and a final cubic-fit placement
// (MolecularMechanics/line_movement.cui).  Molecules never interact, so here a thread block takes
// one work unit (whole molecules whose atoms fit in shared memory) and runs every cycle of every
// molecule in it without leaving the kernel: the unit's parameters and Lennard-Jones tables are
// staged once, each evaluation reuses them, and the per-molecule decisions are made by one thread
// per molecule between block barriers.  Blocks pull units from a device counter, largest first.
//
// Per cycle and molecule, following the reference:
//   1. forces and energy E0 at the line start
//   2. gg = |f_prev|^2, dgg = (f - f_prev) . f, gamma = dgg / gg once the cycle count reaches the
//      steepest-descent cycles (0 before), direction d = f + gamma d (conjugate_gradient.cui:
//      8-140), normalized per molecule
//   3. trial moves of 1 x, then 1.04 or 0.8 x, then 1.03 or 0.85 x the last factor, times the
//      move length, with an energy after each (line_movement.cui:88-126)
//   4. a cubic through the four energies places the molecule and scales the next move length
//      (line_movement.cui:236-336)
// Energies, gg, dgg, the direction norm, gamma and move lengths are FP64 per molecule; per-atom
// arithmetic is FP32 on top of the int64 fixed-point coordinates.  Every per-molecule sum is an
// integer sum or a fixed-order FP64 sum over that molecule's own 32-atom chunks, so a molecule's
// trajectory is bit-identical whichever unit, launch or neighbours it has.
#include <cuda_runtime.h>

#include <type_traits>

#include "line_search.cuh"
#include "unit_eval.cuh"

namespace sb {

namespace {

constexpr int kMolDoubles = 12;

// Per-molecule line-search scalars, kMaxUnitSystems of each
enum MolSlot : int {
  kE0 = 0, kE1, kE2, kE3,      // energies at the line start and the three trial points
  kMv1, kMv2, kMv3,            // cumulative move factors of the trial points
  kMfac,                       // factor of the latest trial move
  kSMove,                      // move length of this cycle (A)
  kLMove,                      // baseline move length of the next cycle (A)
  kInvNorm,                    // 1 / |direction|
  kStep                        // coordinate increment per unit direction, fixed-point units
};

struct MinSmem {
  int msys;       // molecules the carve-out holds (stride of mol)
  double* part;   // three partial sums per 32-slot chunk
  double* mol;    // kMolDoubles x msys
  int* cyc;       // completed cycles
  int* done;      // converged (no further moves)
  int* act;       // moving in the current cycle: not converged, below the cycle limit
};

__host__ __device__ inline size_t minSmemBytes(int max_slots, int max_sys) {
  return alignUp(sizeof(double) * (3 * (max_slots / kTile) + kMolDoubles * max_sys) +
                 sizeof(int) * 3 * max_sys, 16);
}

__device__ MinSmem carveMinSmem(char* base, int max_slots, int max_sys) {
  MinSmem m;
  m.msys = max_sys;
  m.part = reinterpret_cast<double*>(base);
  m.mol = m.part + 3 * (max_slots / kTile);
  m.cyc = reinterpret_cast<int*>(m.mol + kMolDoubles * max_sys);
  m.done = m.cyc + max_sys;
  m.act = m.done + max_sys;
  return m;
}

__device__ __forceinline__ double& molValue(const MinSmem &ms, int slot, int k) {
  return ms.mol[slot * ms.msys + k];
}

// Fixed-order sum of molecule k's chunk partials (component c of three)
__device__ __forceinline__ double moleculeSum(const UnitSmem &s, const MinSmem &ms, int k,
                                              int c) {
  const int c0 = s.slot0[k] / kTile;
  const int c1 = c0 + (s.natom[k] + kTile - 1) / kTile;
  double t = 0.0;
  for (int q = c0; q < c1; q++) {
    t += ms.part[3 * q + c];
  }
  return t;
}

// Total potential energy of unit molecule k from its integer energy slots
__device__ __forceinline__ double moleculeEnergy(const DevSynthesis &d, const UnitSmem &s, int k) {
  long long t = 0;
  for (int q = 0; q < kNrgStride; q++) {
    t += static_cast<long long>(s.nrg[k * kNrgStride + q]);
  }
  return static_cast<double>(t) / static_cast<double>(d.nrg_scale);
}

// Place every slot of the unit at the current coordinates and clear the accumulators
template <class Team>
__device__ void placeUnit(const DevSynthesis &d, const DevMinimizer &m, const UnitSmem &s,
                          const UnitShape &us, const Team &team) {
  for (int e = team.rank(); e < us.nsys * kNrgStride; e += team.size()) {
    s.nrg[e] = 0ull;
  }
  for (int slot = team.rank(); slot < us.nslots; slot += team.size()) {
    const int k = findOwner(s.slot0, us.nsys, slot);
    const int a = slot - s.slot0[k];
    const bool real = a < s.natom[k];
    const int gi = d.atom_start[s.sys[k]] + (real ? a : 0);
    placeSlot(d, s, slot, real, real ? m.xcrd[gi] : 0ll, real ? m.ycrd[gi] : 0ll,
              real ? m.zcrd[gi] : 0ll);
  }
  team.sync();
}

// Move every atom of the molecules with a nonzero step along the direction
template <class Team>
__device__ void moveUnit(const DevSynthesis &d, const DevMinimizer &m, const UnitSmem &s,
                         const MinSmem &ms, const UnitShape &us, const Team &team) {
  for (int slot = team.rank(); slot < us.nslots; slot += team.size()) {
    const int k = findOwner(s.slot0, us.nsys, slot);
    const int a = slot - s.slot0[k];
    const double step = molValue(ms, kStep, k);
    if (a < s.natom[k] && step != 0.0) {
      const int gi = d.atom_start[s.sys[k]] + a;
      m.xcrd[gi] += __double2ll_rn(static_cast<double>(m.xcg[gi]) * step);
      m.ycrd[gi] += __double2ll_rn(static_cast<double>(m.ycg[gi]) * step);
      m.zcrd[gi] += __double2ll_rn(static_cast<double>(m.zcg[gi]) * step);
    }
  }
}

// One line-minimization cycle of every unit molecule that has not converged; with CLASH, the
// four evaluations of a molecule still within m.clash_cycles use softened cores
template <bool HIST, bool CLASH, bool NECK, class Team>
__device__ void minimizationCycle(const DevSynthesis &d, const DevMinimizer &m,
                                  const UnitSmem &s, const MinSmem &ms, const UnitShape &us,
                                  const Team &team) {
  const int lane = threadIdx.x & 31;
  const double inv_fs = 1.0 / static_cast<double>(d.frc_scale);
  const double gpos_scale = 1.0 / d.inv_gpos_scale;

  // 1. forces and energy at the line start (placeUnit ends with the barrier after s.clash)
  if (CLASH && team.rank() < us.nsys) {
    const int k = team.rank();
    s.clash[k] = clashScaled(m.clash_distance, m.clash_ratio, m.clash_cycles, ms.cyc[k]);
  }
  placeUnit(d, m, s, us, team);
  evaluateStaged<true, true, 7, false, CLASH, NECK>(d, s, us, team);

  // 2. gg, dgg and |f|^2 per 32-slot chunk (a chunk never straddles two molecules)
  for (int slot = team.rank(); slot < us.nslots; slot += team.size()) {
    const int k = findOwner(s.slot0, us.nsys, slot);
    const int a = slot - s.slot0[k];
    double gg = 0.0, dgg = 0.0, ff = 0.0;
    if (a < s.natom[k]) {
      const int gi = d.atom_start[s.sys[k]] + a;
      const double fx = static_cast<double>(int63ToLong(s.fx[slot], s.fxo[slot]));
      const double fy = static_cast<double>(int63ToLong(s.fy[slot], s.fyo[slot]));
      const double fz = static_cast<double>(int63ToLong(s.fz[slot], s.fzo[slot]));
      const double px = static_cast<double>(m.xprv[gi]);
      const double py = static_cast<double>(m.yprv[gi]);
      const double pz = static_cast<double>(m.zprv[gi]);
      gg = px * px + py * py + pz * pz;
      dgg = (fx - px) * fx + (fy - py) * fy + (fz - pz) * fz;
      ff = fx * fx + fy * fy + fz * fz;
    }
    gg = warpSumDouble(gg);
    dgg = warpSumDouble(dgg);
    ff = warpSumDouble(ff);
    if (lane == 0) {
      const int q = slot / kTile;
      ms.part[3 * q] = gg;
      ms.part[3 * q + 1] = dgg;
      ms.part[3 * q + 2] = ff;
    }
  }
  team.sync();
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const int sysid = s.sys[k];
    const double gg = moleculeSum(s, ms, k, 0) * inv_fs * inv_fs;
    const double dgg = moleculeSum(s, ms, k, 1) * inv_fs * inv_fs;
    const double ff = moleculeSum(s, ms, k, 2) * inv_fs * inv_fs;
    const double e0 = moleculeEnergy(d, s, k);
    molValue(ms, kE0, k) = e0;
    if (ms.act[k]) {
      const double rms = sqrt(ff / (3.0 * static_cast<double>(s.natom[k])));
      m.rms_force[sysid] = rms;
      if (HIST && ms.cyc[k] < m.hist_stride) {
        m.history[static_cast<size_t>(sysid) * m.hist_stride + ms.cyc[k]] = e0;
      }
      if (m.drms > 0.0 && rms <= m.drms) {
        ms.done[k] = 1;
        ms.act[k] = 0;
      }
    }
    // the reference advances its step counter before the gather (hpc_minimization.cu:470)
    const int step = ms.cyc[k] + 1;
    molValue(ms, kMfac, k) = (step >= m.sd_cycles && gg > 0.0) ? dgg / gg : 0.0;   // gamma
  }
  team.sync();

  // conjugate direction, previous force, |direction|^2
  for (int slot = team.rank(); slot < us.nslots; slot += team.size()) {
    const int k = findOwner(s.slot0, us.nsys, slot);
    const int a = slot - s.slot0[k];
    double msum = 0.0;
    if (a < s.natom[k] && ms.act[k]) {
      const int gi = d.atom_start[s.sys[k]] + a;
      const long long ix = int63ToLong(s.fx[slot], s.fxo[slot]);
      const long long iy = int63ToLong(s.fy[slot], s.fyo[slot]);
      const long long iz = int63ToLong(s.fz[slot], s.fzo[slot]);
      const double gam = molValue(ms, kMfac, k);
      float cx = static_cast<float>(static_cast<double>(ix) * inv_fs);
      float cy = static_cast<float>(static_cast<double>(iy) * inv_fs);
      float cz = static_cast<float>(static_cast<double>(iz) * inv_fs);
      if (fabs(gam) > kVeryTiny) {
        const float g = static_cast<float>(gam);
        cx = fmaf(g, m.xcg[gi], cx);
        cy = fmaf(g, m.ycg[gi], cy);
        cz = fmaf(g, m.zcg[gi], cz);
      }
      m.xcg[gi] = cx;
      m.ycg[gi] = cy;
      m.zcg[gi] = cz;
      m.xprv[gi] = ix;
      m.yprv[gi] = iy;
      m.zprv[gi] = iz;
      msum = static_cast<double>(cx) * cx + static_cast<double>(cy) * cy +
             static_cast<double>(cz) * cz;
    }
    msum = warpSumDouble(msum);
    if (lane == 0) {
      ms.part[3 * (slot / kTile)] = msum;
    }
  }
  team.sync();

  // 3. first trial move: 1 x the move length
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    if (ms.act[k]) {
      const double msum = moleculeSum(s, ms, k, 0);
      const double inv_norm = (msum > 0.0) ? 1.0 / sqrt(msum) : 0.0;
      const double s_move = molValue(ms, kLMove, k);
      molValue(ms, kInvNorm, k) = inv_norm;
      molValue(ms, kSMove, k) = s_move;
      molValue(ms, kMfac, k) = 1.0;
      molValue(ms, kMv1, k) = 1.0;
      molValue(ms, kStep, k) = inv_norm * s_move * gpos_scale;
    }
    else {
      molValue(ms, kStep, k) = 0.0;
    }
  }
  team.sync();
  moveUnit(d, m, s, ms, us, team);
  placeUnit(d, m, s, us, team);
  evaluateStaged<false, true, 7, false, CLASH, NECK>(d, s, us, team);

  // second trial move: 1.04 x after a decrease, else 0.8 x
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const double e1 = moleculeEnergy(d, s, k);
    molValue(ms, kE1, k) = e1;
    if (ms.act[k]) {
      const double mfac = (e1 < molValue(ms, kE0, k)) ? 1.04 : 0.8;
      molValue(ms, kMfac, k) = mfac;
      molValue(ms, kMv2, k) = molValue(ms, kMv1, k) + mfac;
      molValue(ms, kStep, k) = molValue(ms, kInvNorm, k) * mfac * molValue(ms, kSMove, k) *
                               gpos_scale;
    }
  }
  team.sync();
  moveUnit(d, m, s, ms, us, team);
  placeUnit(d, m, s, us, team);
  evaluateStaged<false, true, 7, false, CLASH, NECK>(d, s, us, team);

  // third trial move: the last factor x 1.03 after a decrease, else x 0.85
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const double e2 = moleculeEnergy(d, s, k);
    molValue(ms, kE2, k) = e2;
    if (ms.act[k]) {
      const double mfac = molValue(ms, kMfac, k) * ((e2 < molValue(ms, kE1, k)) ? 1.03 : 0.85);
      molValue(ms, kMfac, k) = mfac;
      molValue(ms, kMv3, k) = molValue(ms, kMv2, k) + mfac;
      molValue(ms, kStep, k) = molValue(ms, kInvNorm, k) * mfac * molValue(ms, kSMove, k) *
                               gpos_scale;
    }
  }
  team.sync();
  moveUnit(d, m, s, ms, us, team);
  placeUnit(d, m, s, us, team);
  evaluateStaged<false, true, 7, false, CLASH, NECK>(d, s, us, team);

  // 4. cubic fit and final placement
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const double e3 = moleculeEnergy(d, s, k);
    if (ms.act[k]) {
      const double ev[4] = {molValue(ms, kE0, k), molValue(ms, kE1, k), molValue(ms, kE2, k), e3};
      const double mv[4] = {0.0, molValue(ms, kMv1, k), molValue(ms, kMv2, k),
                            molValue(ms, kMv3, k)};
      double new_base;
      const double mfac = finalPlacement(ev, mv, &new_base);
      const double s_move = molValue(ms, kSMove, k);
      molValue(ms, kLMove, k) = s_move * new_base;
      molValue(ms, kStep, k) = (fabs(mfac) > kVeryTiny) ?
                               molValue(ms, kInvNorm, k) * mfac * s_move * gpos_scale : 0.0;
      ms.cyc[k] += 1;
    }
    else {
      molValue(ms, kStep, k) = 0.0;
    }
  }
  team.sync();
  moveUnit(d, m, s, ms, us, team);
  team.sync();
}

// Every cycle of one work unit, then its final energies (undamped) and state
template <bool HIST, bool CLASH, bool NECK, class Team>
__device__ void minimizeUnit(const DevSynthesis &d, const DevMinimizer &m, const UnitSmem &s,
                             const MinSmem &ms, int u, int max_lj, int max_sys, int cycles,
                             int final_energy, const Team &team) {
  UnitShape us;
  if (!stageUnitTables(d, s, u, max_lj, &us, team, max_sys)) {
    return;
  }
  for (int slot = team.rank(); slot < us.nslots; slot += team.size()) {
    const int k = findOwner(s.slot0, us.nsys, slot);
    s.prm[slot] = slotParameters(d, s, k, slot - s.slot0[k]);
    if (NECK) {
      s.neck[slot] = slotNeck(d, s, k, slot - s.slot0[k]);
    }
  }
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const int sysid = s.sys[k];
    ms.cyc[k] = m.cycle[sysid];
    ms.done[k] = m.done[sysid];
    molValue(ms, kLMove, k) = m.l_move[sysid];
  }
  team.sync();
  for (int c = 0; c < cycles; c++) {
    int moving = 0;
    if (team.rank() < us.nsys) {
      const int k = team.rank();
      moving = (!ms.done[k] && ms.cyc[k] < m.max_cycles) ? 1 : 0;
      ms.act[k] = moving;
    }
    if (!team.any(moving != 0)) {
      break;
    }
    minimizationCycle<HIST, CLASH, NECK>(d, m, s, ms, us, team);
  }
  if (final_energy) {
    // one more energy evaluation at the final coordinates (hpc_minimization.cu:372-383)
    placeUnit(d, m, s, us, team);
    evaluateStaged<false, true, 7, false, false, NECK>(d, s, us, team);
    for (int e = team.rank(); e < us.nsys * kNrgStride; e += team.size()) {
      d.energies[s.sys[e / kNrgStride] * kNrgStride + (e % kNrgStride)] = s.nrg[e];
    }
    if (HIST && team.rank() < us.nsys) {
      const int k = team.rank();
      if (ms.cyc[k] < m.hist_stride) {
        m.history[static_cast<size_t>(s.sys[k]) * m.hist_stride + ms.cyc[k]] =
          moleculeEnergy(d, s, k);
      }
    }
  }
  if (team.rank() < us.nsys) {
    const int k = team.rank();
    const int sysid = s.sys[k];
    m.cycle[sysid] = ms.cyc[k];
    m.done[sysid] = ms.done[k];
    m.l_move[sysid] = molValue(ms, kLMove, k);
  }
  team.sync();
}

// One thread block per work unit (molecules of up to 2,048 atoms).  The minimizer keeps more
// state live than a single evaluation; two blocks per SM with up to 128 registers a thread run
// faster than four with 64, where the pair loops spill.
template <bool HIST, bool CLASH, bool NECK>
__global__ void __launch_bounds__(256, 2)
kMinimize(const DevSynthesis d, const DevMinimizer m, int unit_begin, int unit_end, int max_lj,
          int cycles, int final_energy) {
  extern __shared__ __align__(16) char smem_raw[];
  const UnitSmem s = carveSmem(smem_raw, d.max_unit_slots, max_lj);
  const MinSmem ms = carveMinSmem(smem_raw + unitSmemBytes(d.max_unit_slots, max_lj),
                                  d.max_unit_slots, kMaxUnitSystems);
  __shared__ int next_unit;
  const BlockTeam team;
  int u = unit_begin + blockIdx.x;
  while (u < unit_end) {
    minimizeUnit<HIST, CLASH, NECK>(d, m, s, ms, u, max_lj, kMaxUnitSystems, cycles,
                                    final_energy, team);
    if (threadIdx.x == 0) {
      next_unit = unit_begin + static_cast<int>(gridDim.x) + atomicAdd(m.queue, 1);
    }
    __syncthreads();
    u = next_unit;
  }
}

__global__ void kMinimizerReset(DevMinimizer m, int nsys, int natom_padded, double dx0) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < natom_padded; i += stride) {
    m.xprv[i] = 0;
    m.yprv[i] = 0;
    m.zprv[i] = 0;
    m.xcg[i] = 0.0f;
    m.ycg[i] = 0.0f;
    m.zcg[i] = 0.0f;
    if (m.xcg64 != nullptr) {
      m.xcg64[i] = 0.0;
      m.ycg64[i] = 0.0;
      m.zcg64[i] = 0.0;
    }
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride) {
    m.l_move[i] = dx0;
    m.cycle[i] = 0;
    m.done[i] = 0;
    m.rms_force[i] = 0.0;
  }
}

}  // namespace

size_t minimizeSmemBytes(int max_slots, int max_lj) {
  return unitSmemBytes(max_slots, max_lj) + minSmemBytes(max_slots, kMaxUnitSystems);
}


cudaError_t launchMinimizerReset(const DevMinimizer &m, const DevSynthesis &d, double dx0,
                                 cudaStream_t stream) {
  const int n = d.natom_padded > d.nsys ? d.natom_padded : d.nsys;
  int blocks = (n + 255) / 256;
  blocks = blocks < 1 ? 1 : (blocks > 1024 ? 1024 : blocks);
  kMinimizerReset<<<blocks, 256, 0, stream>>>(m, d.nsys, d.natom_padded, dx0);
  return cudaGetLastError();
}

// Units [unit_begin, unit_end) for up to `cycles` cycles on at most max_blocks resident blocks.
// m.queue must hold zero when the kernel starts.
cudaError_t launchMinimize(const DevSynthesis &d, const DevMinimizer &m, int unit_begin,
                           int unit_end, int max_lj, int cycles, bool final_energy, int threads,
                           int sm_count, cudaStream_t stream) {
  if (unit_end <= unit_begin) {
    return cudaSuccess;
  }
  const size_t smem = minimizeSmemBytes(d.max_unit_slots, max_lj);
  const bool clash = m.clash_cycles > 0 && (m.clash_distance > 0.0f || m.clash_ratio > 0.0f);
  const bool neck = d.neck_size > 0;
  auto pick = [&](auto hist) {
    constexpr bool H = decltype(hist)::value;
    return neck ? (clash ? kMinimize<H, true, true> : kMinimize<H, false, true>) :
                  (clash ? kMinimize<H, true, false> : kMinimize<H, false, false>);
  };
  auto kern = (m.history != nullptr) ? pick(std::true_type()) : pick(std::false_type());
  cudaError_t err = allowLargeSmem(kern);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) {
    return cudaErrorInvalidConfiguration;
  }
  int blocks = per_sm * sm_count;
  if (blocks > unit_end - unit_begin) {
    blocks = unit_end - unit_begin;
  }
  kern<<<blocks, threads, smem, stream>>>(d, m, unit_begin, unit_end, max_lj, cycles,
                                          final_energy ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace sb
