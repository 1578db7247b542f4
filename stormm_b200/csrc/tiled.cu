// Tiled evaluation of molecules too large for one block's shared memory (the 2,000-5,000-atom
// chains of the large-system workload), with the same pair functors, valence code and integer
// accumulation as the fused kernel: the two paths agree to FP32 rounding (the compiler may
// contract a few operations differently in the two kernels) and each is bit-identical from run
// to run.
//
// Every 32 x 32 tile of every tiled molecule is a warp task.  A warp stages the tile's two atom
// blocks (coordinates as hi / lo float pairs, the pass's payloads) in its own slice of shared
// memory, walks the tile with the fused kernel's functors, and adds its accumulators to global
// integer arrays.  Passes that need the whole molecule finished first (effective radii after
// pass 1, the chain-rule prefactor after pass 2) are separate per-atom kernels.  Warps take
// contiguous runs of tiles, so a warp's energy sums change molecule rarely and flush once per
// molecule.
#include <cuda_runtime.h>

#include "unit_eval.cuh"
#include "tile_tasks.cuh"

namespace sb {

namespace {

constexpr int kStageSlots = 2 * kTile;    // block I in slots 0-31, block J in slots 32-63

// Valence terms reading atoms straight from the global fixed-point arrays and adding forces and
// energies with global integer atomics (one molecule per block row of the launch grid)
struct GlobalValence {
  const DevSynthesis &d;
  const int* bchunk0;
  const int* achunk0;
  const int* dchunk0;
  const int* sys;
  const int* slot0;
  const float2* lj14tab;
  int nt;
  __device__ GlobalValence(const DevSynthesis &d_in, const int* chunks, const int* sys_in,
                           const int* slot0_in, const float2* lj14_in, int nt_in) :
      d(d_in), bchunk0(chunks), achunk0(chunks + 2), dchunk0(chunks + 4), sys(sys_in),
      slot0(slot0_in), lj14tab(lj14_in), nt(nt_in) {}
  __device__ __forceinline__ int chunkBegin() const {
    return (threadIdx.x >> 5) + blockIdx.y * (blockDim.x >> 5);
  }
  __device__ __forceinline__ int chunkStride() const { return (blockDim.x >> 5) * gridDim.y; }
  __device__ __forceinline__ void hilo(int i, float4* a, float4* b) const {
    splitCoordinate(static_cast<double>(d.xcrd[i]) * d.inv_gpos_scale, &a->x, &b->x);
    splitCoordinate(static_cast<double>(d.ycrd[i]) * d.inv_gpos_scale, &a->y, &b->y);
    splitCoordinate(static_cast<double>(d.zcrd[i]) * d.inv_gpos_scale, &a->z, &b->z);
    a->w = 0.0f;
    b->w = 0.0f;
  }
  __device__ __forceinline__ float4 pa(int i) const {
    float4 a, b;
    hilo(i, &a, &b);
    return a;
  }
  __device__ __forceinline__ float4 pb(int i) const {
    float4 a, b;
    hilo(i, &a, &b);
    return b;
  }
  __device__ __forceinline__ float4 prm(int i) const {
    const int ty = d.lj_idx[i];
    return make_float4(d.charge[i], __int_as_float((ty * nt) | (ty << 16)), d.rho[i], d.srho[i]);
  }
  __device__ __forceinline__ float3 delta(int a, int b) const {
    float4 aa, ab, ba, bb;
    hilo(a, &aa, &ab);
    hilo(b, &ba, &bb);
    return pairDelta(aa, ab, ba, bb);
  }
  __device__ __forceinline__ void force(int i, float fx, float fy, float fz, float scale) const {
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.xfrc[i]),
              static_cast<unsigned long long>(__float2ll_rn(fx * scale)));
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.yfrc[i]),
              static_cast<unsigned long long>(__float2ll_rn(fy * scale)));
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.zfrc[i]),
              static_cast<unsigned long long>(__float2ll_rn(fz * scale)));
  }
  __device__ __forceinline__ void energy(int k, int slot, float e, float scale) const {
    const long long v = warpSum(__float2ll_rn(e * scale));
    if ((threadIdx.x & 31) == 0 && v != 0) {
      atomicAdd(&d.energies[sys[k] * kNrgStride + slot], static_cast<unsigned long long>(v));
    }
  }
  __device__ __forceinline__ float2 lj14(int code_i, int code_l, int) const {
    return lj14tab[(code_i & 0xffff) + (code_l >> 16)];
  }
  __device__ __forceinline__ double3 pos64(int i) const {
    return make_double3(static_cast<double>(d.xcrd[i]) * d.inv_gpos_scale,
                        static_cast<double>(d.ycrd[i]) * d.inv_gpos_scale,
                        static_cast<double>(d.zcrd[i]) * d.inv_gpos_scale);
  }
  __device__ __forceinline__ void force64(int i, double fx, double fy, double fz,
                                          float scale) const {
    const double s = static_cast<double>(scale);
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.xfrc[i]),
              static_cast<unsigned long long>(__double2ll_rn(fx * s)));
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.yfrc[i]),
              static_cast<unsigned long long>(__double2ll_rn(fy * s)));
    atomicAdd(reinterpret_cast<unsigned long long*>(&d.zfrc[i]),
              static_cast<unsigned long long>(__double2ll_rn(fz * s)));
  }
  __device__ __forceinline__ void energy64(int k, int slot, double e, float scale) const {
    const long long v = warpSum(__double2ll_rn(e * static_cast<double>(scale)));
    if ((threadIdx.x & 31) == 0 && v != 0) {
      atomicAdd(&d.energies[sys[k] * kNrgStride + slot], static_cast<unsigned long long>(v));
    }
  }
  __device__ __forceinline__ float2 clash(int k) const {
    const int cycle = (d.clash_cycle != nullptr) ? d.clash_cycle[sys[k]] : -1;
    return clashScaled(d.clash_distance, d.clash_ratio, d.clash_cycles, cycle);
  }
};

// Valence terms of tiled molecule blockIdx.x (plus mol_begin), chunks spread over blockIdx.y
template <bool FORCE, bool ENERGY, bool CLASH>
__global__ void __launch_bounds__(256)
kTiledValence(const DevSynthesis d, const DevTiled t, int mol_begin) {
  __shared__ int sys[1];
  __shared__ int slot0[1];
  __shared__ int chunks[6];   // bond, angle, dihedral chunk prefix sums (0, count) each
  const int m = mol_begin + blockIdx.x;
  if (threadIdx.x == 0) {
    const int s = t.systems[m];
    sys[0] = s;
    slot0[0] = d.atom_start[s];
    chunks[0] = 0;
    chunks[1] = (d.bond_start[s + 1] - d.bond_start[s] + 31) / 32;
    chunks[2] = 0;
    chunks[3] = (d.angl_start[s + 1] - d.angl_start[s] + 31) / 32;
    chunks[4] = 0;
    chunks[5] = (d.dihe_start[s + 1] - d.dihe_start[s] + 31) / 32;
  }
  __syncthreads();
  const int s = sys[0];
  const GlobalValence v(d, chunks, sys, slot0, d.ljab14 + d.lj_start[s], d.lj_ntypes[s]);
  valenceTerms<FORCE, ENERGY, GlobalValence, CLASH>(d, v, 1);
}

// Stage one tile's atom blocks into a warp's slice: block I in slots 0-31, block J in 32-63
// (a diagonal tile stages block I only).  PASS 1 and 3 carry s * rho and rho, PASS 2 the charge
// and the effective radius; padding slots get the fused kernel's zero-contribution values.
template <int PASS, bool GB>
__device__ __forceinline__ void stageTile(const DevSynthesis &d, const DevTiled &t,
                                          const UnitSmem &v, int sysid, int I, int J, bool diag,
                                          int lane) {
  const int natom = d.atom_count[sysid];
  const int base = d.atom_start[sysid];
  const int nt = d.lj_ntypes[sysid];
  for (int half = 0; half < (diag ? 1 : 2); half++) {
    const int a = (half == 0 ? I : J) * kTile + lane;
    const int slot = half * kTile + lane;
    float4 pa, pb, prm;
    float2 gbv = make_float2(1.0f, 0.0f);
    if (a < natom) {
      const int gi = base + a;
      pa.w = 0.0f;
      pb.w = 0.0f;
      splitCoordinate(static_cast<double>(d.xcrd[gi]) * d.inv_gpos_scale, &pa.x, &pb.x);
      splitCoordinate(static_cast<double>(d.ycrd[gi]) * d.inv_gpos_scale, &pa.y, &pb.y);
      splitCoordinate(static_cast<double>(d.zcrd[gi]) * d.inv_gpos_scale, &pa.z, &pb.z);
      const int ty = d.lj_idx[gi];
      prm = make_float4(d.charge[gi], __int_as_float((ty * nt) | (ty << 16)), d.rho[gi],
                        d.srho[gi]);
      if (PASS == 2) {
        pa.w = prm.x;
        gbv.y = prm.y;      // the Lennard-Jones code, where pass 2 reads it
        if (GB) {
          const float r = t.radius[gi];
          pb.w = r;
          gbv.x = 1.0f / r;
        }
        else {
          pb.w = prm.z;
        }
      }
      else {
        pa.w = prm.w;
        pb.w = prm.z;
        if (PASS == 3) {
          gbv.y = t.sde[gi];
        }
      }
    }
    else {
      pa = make_float4(5000.0f + 16.0f * static_cast<float>(slot), 0.0f, 0.0f, 0.0f);
      pb = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
      prm = make_float4(0.0f, __int_as_float(0), 1.0f, 0.0f);
    }
    v.pa[slot] = pa;
    v.pb[slot] = pb;
    v.prm[slot] = prm;
    v.gbv[slot] = gbv;
    v.neck[slot] = (d.neck_size > 0 && a < natom) ? d.neck_idx[base + a] : 0;
  }
  __syncwarp();
}

__device__ __forceinline__ UnitSmem warpView(float4* pa, float4* pb, float4* prm, float2* gbv,
                                             int* neck, const float2* lj) {
  UnitSmem v{};
  const int w = threadIdx.x >> 5;
  v.pa = pa + w * kStageSlots;
  v.pb = pb + w * kStageSlots;
  v.prm = prm + w * kStageSlots;
  v.gbv = gbv + w * kStageSlots;
  v.neck = neck + w * kStageSlots;
  v.lj = const_cast<float2*>(lj);
  return v;
}

__device__ __forceinline__ void addGlobal(long long* acc, float v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(acc),
            static_cast<unsigned long long>(__float2ll_rn(v)));
}

// GB pass 1 over tiles [tile_begin, tile_end)
template <bool NECK>
__global__ void __launch_bounds__(256, 4)
kTiledRadii(const DevSynthesis d, const DevTiled t, int tile_begin, int tile_end) {
  __shared__ float4 pa[kTiledWarps * kStageSlots], pb[kTiledWarps * kStageSlots];
  __shared__ float4 prm[kTiledWarps * kStageSlots];
  __shared__ float2 gbv[kTiledWarps * kStageSlots];
  __shared__ int neck[kTiledWarps * kStageSlots];
  const int lane = threadIdx.x & 31;
  const float ps = static_cast<float>(1 << kPsiBits);
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  const UnitSmem v = warpView(pa, pb, prm, gbv, neck, d.ljab);
  RadiiPass2<NECK> p(v, d);
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    stageTile<1, true>(d, t, v, sysid, I, J, ti.diag, lane);
    p.begin(lane);
    walkTile2(p, ti, lane);
    const int base = d.atom_start[sysid];
    if (lane < ti.ni) {
      addGlobal(&t.psi_acc[base + I * kTile + lane], p.psi_i * ps);
    }
    const int jl = traveledAtom2(ti, lane);
    if (jl < ti.nj) {
      addGlobal(&t.psi_acc[base + J * kTile + jl], p.psi_j1 * ps);
    }
    __syncwarp();
  }
}

// Pass 2 (Coulomb + Lennard-Jones and GB pair terms) over tiles [tile_begin, tile_end)
template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH>
__global__ void __launch_bounds__(256, 4)
kTiledPair(const DevSynthesis d, const DevTiled t, int tile_begin, int tile_end) {
  __shared__ float4 pa[kTiledWarps * kStageSlots], pb[kTiledWarps * kStageSlots];
  __shared__ float4 prm[kTiledWarps * kStageSlots];
  __shared__ float2 gbv[kTiledWarps * kStageSlots];
  __shared__ int neck[kTiledWarps * kStageSlots];
  const int lane = threadIdx.x & 31;
  const float fs = d.frc_scale;
  const float es = d.nrg_scale;
  const float ds = static_cast<float>(1 << kDeijdaBits);
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  long long acc_elec = 0, acc_vdw = 0, acc_gb = 0;
  int acc_sys = -1;
  auto flush = [&]() {
    // per-tile energies rounded to the output grid (tileEnergy), the same value in every lane
    if (lane == 0 && acc_sys >= 0) {
      if (NB) {
        atomicAdd(&d.energies[acc_sys * kNrgStride + kElec],
                  static_cast<unsigned long long>(acc_elec));
        atomicAdd(&d.energies[acc_sys * kNrgStride + kVdw],
                  static_cast<unsigned long long>(acc_vdw));
      }
      if (GB) {
        atomicAdd(&d.energies[acc_sys * kNrgStride + kGb], static_cast<unsigned long long>(acc_gb));
      }
    }
    acc_elec = acc_vdw = acc_gb = 0;
  };
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    if (ENERGY && sysid != acc_sys) {
      flush();
      acc_sys = sysid;
    }
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    const UnitSmem v = warpView(pa, pb, prm, gbv, neck, d.ljab + d.lj_start[sysid]);
    stageTile<2, GB>(d, t, v, sysid, I, J, ti.diag, lane);
    unsigned mask = 0u;
    if (NB) {
      const int midx = d.tile_mask_idx[d.tile_start[sysid] + ti.local];
      if (midx != 0) {
        mask = __ldg(&d.mask_pool[static_cast<size_t>(midx) * 32 + lane]);
      }
    }
    PairPass<FORCE, ENERGY, NB, GB, CLASH> p(v, d.kappa, d.inv_dielectric);
    float2 clash = make_float2(0.0f, 0.0f);
    if (CLASH) {
      const int cycle = (d.clash_cycle != nullptr) ? d.clash_cycle[sysid] : -1;
      clash = clashScaled(d.clash_distance, d.clash_ratio, d.clash_cycles, cycle);
    }
    p.begin(lane, mask, clash);
    walkTile(p, ti, lane);
    const int base = d.atom_start[sysid];
    if (FORCE) {
      if (lane < ti.ni) {
        const int gi = base + I * kTile + lane;
        addGlobal(&d.xfrc[gi], p.fxi * fs);
        addGlobal(&d.yfrc[gi], p.fyi * fs);
        addGlobal(&d.zfrc[gi], p.fzi * fs);
        if (GB) {
          addGlobal(&t.de_acc[gi], p.dei * ds);
        }
      }
      const int jl = traveledAtom(ti, lane);
      if (jl < ti.nj) {
        const int gj = base + J * kTile + jl;
        addGlobal(&d.xfrc[gj], p.fxj * fs);
        addGlobal(&d.yfrc[gj], p.fyj * fs);
        addGlobal(&d.zfrc[gj], p.fzj * fs);
        if (GB) {
          addGlobal(&t.de_acc[gj], p.dej * ds);
        }
      }
    }
    if (ENERGY) {
      if (NB) {
        acc_elec += tileEnergy(p.t_elec, es);
        acc_vdw += tileEnergy(p.t_vdw, es);
      }
      if (GB) {
        acc_gb += tileEnergy(p.t_gb, es);
      }
    }
    __syncwarp();
  }
  if (ENERGY) {
    flush();
  }
}

// Pass 3 (radius chain-rule forces) over tiles [tile_begin, tile_end)
template <bool NECK>
__global__ void __launch_bounds__(256, 4)
kTiledDeriv(const DevSynthesis d, const DevTiled t, int tile_begin, int tile_end) {
  __shared__ float4 pa[kTiledWarps * kStageSlots], pb[kTiledWarps * kStageSlots];
  __shared__ float4 prm[kTiledWarps * kStageSlots];
  __shared__ float2 gbv[kTiledWarps * kStageSlots];
  __shared__ int neck[kTiledWarps * kStageSlots];
  const int lane = threadIdx.x & 31;
  const float fs = d.frc_scale;
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  const UnitSmem v = warpView(pa, pb, prm, gbv, neck, d.ljab);
  DerivPass<NECK> p(v, d);
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    stageTile<3, true>(d, t, v, sysid, I, J, ti.diag, lane);
    p.begin(lane);
    walkTile(p, ti, lane);
    const int base = d.atom_start[sysid];
    if (lane < ti.ni) {
      const int gi = base + I * kTile + lane;
      addGlobal(&d.xfrc[gi], p.fxi * fs);
      addGlobal(&d.yfrc[gi], p.fyi * fs);
      addGlobal(&d.zfrc[gi], p.fzi * fs);
    }
    const int jl = traveledAtom(ti, lane);
    if (jl < ti.nj) {
      const int gj = base + J * kTile + jl;
      addGlobal(&d.xfrc[gj], p.fxj * fs);
      addGlobal(&d.yfrc[gj], p.fyj * fs);
      addGlobal(&d.zfrc[gj], p.fzj * fs);
    }
    __syncwarp();
  }
}

// Effective radii and GB self terms of the tiled atoms [atom_begin, atom_end) (padded
// positions; a warp's 32 positions always belong to one molecule)
template <bool FORCE, bool ENERGY, bool WS>
__global__ void __launch_bounds__(256)
kTiledAtoms(const DevSynthesis d, const DevTiled t, int atom_begin, int atom_end) {
  const float inv_ps = 1.0f / static_cast<float>(1 << kPsiBits);
  const float ds = static_cast<float>(1 << kDeijdaBits);
  for (int q = atom_begin + blockIdx.x * blockDim.x + threadIdx.x; q < atom_end;
       q += gridDim.x * blockDim.x) {
    int sysid, a;
    const int gi = tiledAtom(d, t, q, &sysid, &a);
    float e_self = 0.0f;
    float egbi = 1.0f;
    if (a < d.atom_count[sysid]) {
      const double psi = static_cast<double>(t.psi_acc[gi]) * static_cast<double>(inv_ps);
      egbi = effectiveRadius(d, gi, psi);
      float self_de;
      e_self = gbSelfTerm(d, d.charge[gi], egbi, &self_de);
      if (FORCE) {
        addGlobal(&t.de_acc[gi], self_de * ds);
      }
      if (WS) {
        d.born_radii[gi] = egbi;
        d.psi[gi] = __double2ll_rn(static_cast<double>(psi) * d.psi_out_scale);
        d.psi_ovrf[gi] = 0;
      }
    }
    t.radius[gi] = egbi;
    if (ENERGY) {
      const long long v = warpSum(__float2ll_rn(e_self * d.nrg_scale));
      if ((threadIdx.x & 31) == 0 && v != 0) {
        atomicAdd(&d.energies[sysid * kNrgStride + kGb], static_cast<unsigned long long>(v));
      }
    }
  }
}

// Chain-rule prefactor of the tiled atoms' dE/dR sums
template <bool WS>
__global__ void __launch_bounds__(256)
kTiledChain(const DevSynthesis d, const DevTiled t, int atom_begin, int atom_end) {
  const float inv_ds = 1.0f / static_cast<float>(1 << kDeijdaBits);
  const float inv_ps = 1.0f / static_cast<float>(1 << kPsiBits);
  for (int q = atom_begin + blockIdx.x * blockDim.x + threadIdx.x; q < atom_end;
       q += gridDim.x * blockDim.x) {
    int sysid, a;
    const int gi = tiledAtom(d, t, q, &sysid, &a);
    float sde = 0.0f;
    if (a < d.atom_count[sysid]) {
      sde = static_cast<float>(t.de_acc[gi]) * inv_ds;
      if (d.igb != 1) {
        const double psi = static_cast<double>(t.psi_acc[gi]) * static_cast<double>(inv_ps);
        sde *= obcChainFactor(d, gi, psi);
      }
      if (WS) {
        d.sumdeijda[gi] = __double2ll_rn(static_cast<double>(sde) * d.psi_out_scale);
        d.sumdeijda_ovrf[gi] = 0;
      }
    }
    t.sde[gi] = sde;
  }
}

}  // namespace

// All requested terms of tiled molecules [mol_begin, mol_end).  psi_acc and de_acc of those
// molecules' atoms must be zero on entry (the caller clears them on the stream).
cudaError_t launchTiled(const DevSynthesis &d, const DevTiled &t, const int* h_tile_prefix,
                        const int* h_atom_prefix, int mol_begin, int mol_end, int terms,
                        bool force, bool energy, bool workspace, int sm_count,
                        cudaStream_t stream, bool clash) {
  if (mol_end <= mol_begin) {
    return cudaSuccess;
  }
  const bool vale = (terms & 1) != 0;
  const bool nb = (terms & 2) != 0;
  const bool gb = ((terms & 4) != 0) && d.igb != 0;
  const int tb = h_tile_prefix[mol_begin], te = h_tile_prefix[mol_end];
  const int ab = h_atom_prefix[mol_begin], ae = h_atom_prefix[mol_end];
  const int tgrid = tileGrid(te - tb, sm_count);
  const int agrid = atomGrid(ae - ab, sm_count);
  const int nmol = mol_end - mol_begin;
  if (vale) {
    const dim3 vgrid(nmol, 4);
#define SB_VALE(C)                                                                             \
    if (force && energy) kTiledValence<true, true, C><<<vgrid, 256, 0, stream>>>(d, t, mol_begin); \
    else if (force) kTiledValence<true, false, C><<<vgrid, 256, 0, stream>>>(d, t, mol_begin);   \
    else kTiledValence<false, true, C><<<vgrid, 256, 0, stream>>>(d, t, mol_begin);
    if (clash) { SB_VALE(true) }
    else { SB_VALE(false) }
#undef SB_VALE
  }
  if (gb) {
    if (d.neck_size > 0) kTiledRadii<true><<<tgrid, 256, 0, stream>>>(d, t, tb, te);
    else kTiledRadii<false><<<tgrid, 256, 0, stream>>>(d, t, tb, te);
#define SB_ATOMS(F, E) \
    if (workspace) kTiledAtoms<F, E, true><<<agrid, 256, 0, stream>>>(d, t, ab, ae); \
    else kTiledAtoms<F, E, false><<<agrid, 256, 0, stream>>>(d, t, ab, ae);
    if (force && energy) { SB_ATOMS(true, true) }
    else if (force) { SB_ATOMS(true, false) }
    else { SB_ATOMS(false, true) }
#undef SB_ATOMS
  }
  if (nb || gb) {
#define SB_PAIR(F, E, C)                                                                      \
    if (nb && gb) kTiledPair<F, E, true, true, C><<<tgrid, 256, 0, stream>>>(d, t, tb, te);    \
    else if (nb) kTiledPair<F, E, true, false, C><<<tgrid, 256, 0, stream>>>(d, t, tb, te);   \
    else kTiledPair<F, E, false, true, false><<<tgrid, 256, 0, stream>>>(d, t, tb, te);
    if (clash) {
      if (force && energy) { SB_PAIR(true, true, true) }
      else if (force) { SB_PAIR(true, false, true) }
      else { SB_PAIR(false, true, true) }
    }
    else {
      if (force && energy) { SB_PAIR(true, true, false) }
      else if (force) { SB_PAIR(true, false, false) }
      else { SB_PAIR(false, true, false) }
    }
#undef SB_PAIR
  }
  if (gb && force) {
    if (workspace) kTiledChain<true><<<agrid, 256, 0, stream>>>(d, t, ab, ae);
    else kTiledChain<false><<<agrid, 256, 0, stream>>>(d, t, ab, ae);
    if (d.neck_size > 0) kTiledDeriv<true><<<tgrid, 256, 0, stream>>>(d, t, tb, te);
    else kTiledDeriv<false><<<tgrid, 256, 0, stream>>>(d, t, tb, te);
  }
  return cudaGetLastError();
}

}  // namespace sb
