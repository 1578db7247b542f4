// Fused batched evaluation of valence, Coulomb + Lennard-Jones and Generalized Born terms.
//
// One thread block evaluates one work unit at a time: a group of whole molecules whose atoms
// fit in shared memory.  Everything a molecule needs stays on chip for the whole evaluation:
//
//   stage       int64 fixed-point coordinates -> (hi, lo) float pairs, per-atom parameters,
//               per-molecule Lennard-Jones tables
//   valence     bonds, angles, dihedrals and their attached 1-4 pairs
//               (Potential/valence_potential.tpp:9-1420 restated for FP32)
//   GB pass 1   Born-radius descreening sums psi_i over all pairs, both directions
//               (Potential/nonbonded_potential.tpp:511-728)
//   radii       effective radii, GB self energy and its dE/dR (nonbonded_potential.tpp:730-805)
//   pass 2      Coulomb + Lennard-Jones on non-excluded pairs, GB pair energy and force, dE/dR
//               sums (nonbonded_potential.tpp:8-425, 808-975); with CLASH, softened cores
//               (soft_core_potentials.tpp) for molecules given a clash distance or ratio
//   chain rule  OBC prefactor on dE/dR (nonbonded_potential.tpp:982-1021)
//   pass 3      radius chain-rule forces (nonbonded_potential.tpp:1022-1290)
//   commit      forces into the int64 + int32-overflow arrays, energies into per-system slots
//
// Pair passes walk 32 x 32 tiles of a molecule's lower triangle, one tile per warp.  Lane l
// holds atom i = I*32 + l in registers; j atoms rotate through the lanes (lane l meets atom
// (l + k) mod 32 of block J at step k) and j-side accumulators travel with a shuffle per step.
// Diagonal tiles take 16 steps, the last one on half the lanes, so every pair is visited once.
// Forces, psi and dE/dR leave registers once per tile through integer shared-memory atomics,
// so every sum is independent of scheduling and the results are bit-identical run to run.
//
// Shared memory per atom slot: pos_a = (x_hi, y_hi, z_hi, w1) and pos_b = (x_lo, y_lo, z_lo, w2)
// feed the pair passes with two 16-byte loads per partner; w1 / w2 carry what the pass needs
// (pass 1 and 3: s*rho and rho; pass 2: charge and effective radius).  prm holds the static
// per-atom values, gbv the reciprocal effective radius and the chain-rule dE/dR.
#include "unit_eval.cuh"

namespace sb {

// Dynamic shared memory needed for a work unit of max_slots atom slots and max_lj table entries
size_t fusedSmemBytes(int max_slots, int max_lj) { return unitSmemBytes(max_slots, max_lj); }

// ------------------------------------------------------------------------------------------------
// The fused kernel: stage, evaluate, commit, one work unit at a time
// ------------------------------------------------------------------------------------------------
template <bool FORCE, bool ENERGY, int TERMS, bool CLASH, bool NECK>
__device__ __forceinline__ void evalFusedUnits(const DevSynthesis &d, int unit_begin,
                                               int unit_end, int max_lj) {
  extern __shared__ __align__(16) char smem_raw[];
  const UnitSmem s = carveSmem(smem_raw, d.max_unit_slots, max_lj);
  for (int u = unit_begin + blockIdx.x; u < unit_end; u += gridDim.x) {
    UnitShape us;
    if (!stageUnitTables(d, s, u, max_lj, &us, BlockTeam())) {
      continue;
    }
    for (int e = threadIdx.x; e < us.nsys * kNrgStride; e += blockDim.x) {
      s.nrg[e] = 0ull;
    }
    if (CLASH) {
      for (int k = threadIdx.x; k < us.nsys; k += blockDim.x) {
        const int cycle = (d.clash_cycle != nullptr) ? d.clash_cycle[s.sys[k]] : -1;
        s.clash[k] = clashScaled(d.clash_distance, d.clash_ratio, d.clash_cycles, cycle);
      }
    }
    // stage atoms (a warp's 32 consecutive slots always belong to one molecule)
    for (int slot = threadIdx.x; slot < us.nslots; slot += blockDim.x) {
      const int k = findOwner(s.slot0, us.nsys, slot);
      const int a = slot - s.slot0[k];
      s.prm[slot] = slotParameters(d, s, k, a);
      if (NECK) {
        s.neck[slot] = slotNeck(d, s, k, a);
      }
      const bool real = a < s.natom[k];
      const int gi = d.atom_start[s.sys[k]] + (real ? a : 0);
      placeSlot(d, s, slot, real, real ? d.xcrd[gi] : 0ll, real ? d.ycrd[gi] : 0ll,
                real ? d.zcrd[gi] : 0ll);
    }
    __syncthreads();
    evaluateStaged<FORCE, ENERGY, TERMS, true, CLASH, NECK>(d, s, us, BlockTeam());

    // commit forces (each atom belongs to exactly one unit) and energies
    if (FORCE) {
      for (int slot = threadIdx.x; slot < us.nslots; slot += blockDim.x) {
        const int k = findOwner(s.slot0, us.nsys, slot);
        const int a = slot - s.slot0[k];
        if (a >= s.natom[k]) continue;
        const int gi = d.atom_start[s.sys[k]] + a;
        addInt95(int63ToLong(s.fx[slot], s.fxo[slot]), &d.xfrc[gi], &d.xfrc_ovrf[gi]);
        addInt95(int63ToLong(s.fy[slot], s.fyo[slot]), &d.yfrc[gi], &d.yfrc_ovrf[gi]);
        addInt95(int63ToLong(s.fz[slot], s.fzo[slot]), &d.zfrc[gi], &d.zfrc_ovrf[gi]);
      }
    }
    if (ENERGY) {
      for (int e = threadIdx.x; e < us.nsys * kNrgStride; e += blockDim.x) {
        const unsigned long long v = s.nrg[e];
        if (v != 0ull) {
          atomicAdd(&d.energies[s.sys[e / kNrgStride] * kNrgStride + (e % kNrgStride)], v);
        }
      }
    }
    __syncthreads();
  }
}

template <bool FORCE, bool ENERGY, int TERMS, bool CLASH, bool NECK>
__global__ void __launch_bounds__(256, 4)
kEvalFused(const DevSynthesis d, int unit_begin, int unit_end, int max_lj) {
  evalFusedUnits<FORCE, ENERGY, TERMS, CLASH, NECK>(d, unit_begin, unit_end, max_lj);
}

// The same with 512 threads a block: twice the warps per work unit, for launches of too few
// units to fill the GPU with 256-thread blocks (a small batch, or its large molecules)
template <bool FORCE, bool ENERGY, int TERMS, bool CLASH, bool NECK>
__global__ void __launch_bounds__(512, 2)
kEvalFusedWide(const DevSynthesis d, int unit_begin, int unit_end, int max_lj) {
  evalFusedUnits<FORCE, ENERGY, TERMS, CLASH, NECK>(d, unit_begin, unit_end, max_lj);
}

// Host-side launcher (called from the C++ layer)
cudaError_t launchEvalFused(const DevSynthesis &d, int unit_begin, int unit_end, int max_lj,
                            int terms, bool force, bool energy, int blocks, int threads,
                            cudaStream_t stream, bool clash) {
  const size_t smem = fusedSmemBytes(d.max_unit_slots, max_lj);
  // softened cores change only Coulomb, Lennard-Jones and 1-4 terms, the neck term only GB
  clash = clash && (terms & 3) != 0;
  const bool neck = d.neck_size > 0 && (terms & 4) != 0;
  // 512-thread blocks exist for evaluations of all terms only
  if (threads > 256 && terms != 7) {
    threads = 256;
  }
  if (threads != 512 && (threads < 64 || threads > 256 || threads % 32 != 0)) {
    return cudaErrorInvalidValue;
  }
#define SB_PICK(K, F, E, T)                                                                     \
    (neck ? (clash ? K<F, E, T, ((T) & 3) != 0, ((T) & 4) != 0> :                               \
                     K<F, E, T, false, ((T) & 4) != 0>) :                                       \
            (clash ? K<F, E, T, ((T) & 3) != 0, false> : K<F, E, T, false, false>))
#define SB_GO(KERN)                                                                             \
  {                                                                                             \
    auto kern = KERN;                                                                           \
    const cudaError_t err = allowLargeSmem(kern);                                               \
    if (err != cudaSuccess) return err;                                                         \
    kern<<<blocks, threads, smem, stream>>>(d, unit_begin, unit_end, max_lj);                   \
    return cudaGetLastError();                                                                  \
  }
#define SB_LAUNCH(F, E, T)                                                                      \
  {                                                                                             \
    if constexpr ((T) == 7) {                                                                   \
      if (threads > 256) SB_GO(SB_PICK(kEvalFusedWide, F, E, T))                                \
    }                                                                                           \
    SB_GO(SB_PICK(kEvalFused, F, E, T))                                                         \
  }
#define SB_TERMS(F, E)                                  \
  switch (terms) {                                      \
  case 1: SB_LAUNCH(F, E, 1)                            \
  case 2: SB_LAUNCH(F, E, 2)                            \
  case 3: SB_LAUNCH(F, E, 3)                            \
  case 4: SB_LAUNCH(F, E, 4)                            \
  case 5: SB_LAUNCH(F, E, 5)                            \
  case 6: SB_LAUNCH(F, E, 6)                            \
  case 7: SB_LAUNCH(F, E, 7)                            \
  default: return cudaErrorInvalidValue;                \
  }
  if (force && energy) {
    SB_TERMS(true, true)
  }
  else if (force) {
    SB_TERMS(true, false)
  }
  else if (energy) {
    SB_TERMS(false, true)
  }
  return cudaErrorInvalidValue;
#undef SB_TERMS
#undef SB_LAUNCH
#undef SB_GO
#undef SB_PICK
}

}  // namespace sb

