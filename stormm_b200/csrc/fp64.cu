// FP64-arithmetic evaluation: the reference's PrecisionModel::DOUBLE counterpart of the FP32
// path, for error and throughput comparisons (STORMM keeps double-precision parameter kits
// beside the single-precision ones, Synthesis/atomgraph_synthesis.h, and runs ktgd* kernels on
// them).  Every molecule is evaluated tile by tile on the tiled path's task list (tile_tasks.cuh):
// a warp stages a tile's two atom blocks as doubles in shared memory and walks the tile with the
// same lane rotation as the FP32 kernels, in double arithmetic from double parameters, with the
// reference's four-case HCT integral and derivative (nonbonded_potential.tpp:589-640,
// 1116-1165).  Accumulation stays integer: forces and energies in the synthesis' fixed-point
// formats, psi and dE/dR at 2^40 (finer than the FP32 path's, so the integer grid does not limit
// the FP64 result), hence results are bit-identical run to run.  Valence terms are one thread per
// term (Potential/valence_potential.tpp:9-578, 1288-1420).
#include <cuda_runtime.h>

#include "stormm_b200.h"
#include "tile_tasks.cuh"

namespace sb {

namespace {

constexpr int kAcc64Bits = 40;                 // fixed-point bits of psi and dE/dR here
constexpr double kAcc64Scale = static_cast<double>(1ull << kAcc64Bits);
constexpr double kInvAcc64Scale = 1.0 / kAcc64Scale;
constexpr int kSlots64 = 2 * kTile;            // a warp's staged slots: block I, then block J

// Constants/generalized_born.h:21-44, 123
constexpr double kTaylorA64 = 1.0 / 3.0;
constexpr double kTaylorB64 = 2.0 / 5.0;
constexpr double kTaylorC64 = 3.0 / 7.0;
constexpr double kTaylorD64 = 4.0 / 9.0;
constexpr double kTaylorDD64 = 5.0 / 11.0;
constexpr double kTaylorE64 = 4.0 / 3.0;
constexpr double kTaylorF64 = 12.0 / 5.0;
constexpr double kTaylorG64 = 24.0 / 7.0;
constexpr double kTaylorH64 = 40.0 / 9.0;
constexpr double kTaylorHH64 = 60.0 / 11.0;
constexpr double kGbKscale64 = 0.73;
// Math/rounding.tpp (the arcsine route of a dihedral near 0 or pi)
constexpr double kNearToOne = 0.999999992549419403076171875;
constexpr double kPi64 = 3.14159265358979323846;

// A warp's staged tile: pa = (x, y, z, w1), pb = (w2, w3, -, -), code = Lennard-Jones type
// (pass 2) or neck GB index (passes 1 and 3)
struct Stage64 {
  double4* pa;
  double4* pb;
  int* code;
};

__device__ __forceinline__ Stage64 warpStage(double4* pa, double4* pb, int* code) {
  const int w = threadIdx.x >> 5;
  return Stage64{pa + w * kSlots64, pb + w * kSlots64, code + w * kSlots64};
}

// Neck GB terms in FP64 (nonbonded_potential.tpp:678-702, 1219-1245); size 0: not a neck model
struct Neck64 {
  const double* sep;
  const double* val;
  int size;
  double scale;
  double reach;    // 2 offset + cutoff
  __device__ Neck64(const DevSynthesis &d, const DevPrecise &p) :
      sep(p.neck_sep), val(p.neck_val), size(d.neck_size), scale(p.neck_scale),
      reach(2.0 * p.gb_offset + p.neck_cut) {}
  __device__ __forceinline__ double term(int ni, int nj, double r, double* deriv) const {
    const int t = size * nj + ni;
    const double m = r - sep[t];
    const double m2 = m * m;
    const double den = 1.0 + m2 + 0.3 * m2 * m2 * m2;
    *deriv = ((2.0 * m + 1.8 * m2 * m2 * m) * val[t] * scale) / (den * den * r);
    return scale * val[t] / den;
  }
};

__device__ __forceinline__ void addFixed(long long* acc, double v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(acc),
            static_cast<unsigned long long>(__double2ll_rn(v)));
}

__device__ __forceinline__ long long warpSum64(long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// Add a per-lane energy (kcal/mol) of system sysid into its slot
__device__ __forceinline__ void warpEnergy64(const DevSynthesis &d, int sysid, int slot,
                                             double e) {
  const long long v = warpSum64(__double2ll_rn(e * static_cast<double>(d.nrg_scale)));
  if ((threadIdx.x & 31) == 0 && v != 0) {
    atomicAdd(&d.energies[static_cast<size_t>(sysid) * kNrgStride + slot],
              static_cast<unsigned long long>(v));
  }
}

// ------------------------------------------------------------------------------------------------
// HCT descreening and its radial derivative, the reference's case by case forms
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double hctIntegral64(double r, double rho, double sj) {
  const double r2 = r * r;
  const double invr = 1.0 / r;
  const double sj2 = sj * sj;
  if (r > 4.0 * sj) {
    const double invr2 = invr * invr;
    const double t = sj2 * invr2;
    return sj * t * invr2 *
           (kTaylorA64 + t * (kTaylorB64 + t * (kTaylorC64 + t * (kTaylorD64 + t * kTaylorDD64))));
  }
  if (r > rho + sj) {
    return 0.5 * (sj / (r2 - sj2) + 0.5 * invr * log((r - sj) / (r + sj)));
  }
  if (r > fabs(rho - sj)) {
    const double inv_rho = 1.0 / rho;
    const double theta = 0.5 * inv_rho * invr * (r2 + rho * rho - sj2);
    const double uij = 1.0 / (r + sj);
    return 0.25 * (inv_rho * (2.0 - theta) - uij + invr * log(rho * uij));
  }
  if (rho < sj) {
    return 0.5 * (sj / (r2 - sj2) + 2.0 / rho + 0.5 * invr * log((sj - r) / (sj + r)));
  }
  return 0.0;
}

// -(1/r) dI/dr
__device__ __forceinline__ double hctDerivative64(double r, double rho, double sj) {
  const double r2 = r * r;
  const double invr = 1.0 / r;
  const double invr2 = invr * invr;
  const double sj2 = sj * sj;
  if (r > 4.0 * sj) {
    const double t = sj2 * invr2;
    return t * sj * invr2 * invr2 *
           (kTaylorE64 + t * (kTaylorF64 + t * (kTaylorG64 + t * (kTaylorH64 + t * kTaylorHH64))));
  }
  if (r > rho + sj) {
    const double temp1 = 1.0 / (r2 - sj2);
    return temp1 * sj * (-0.5 * invr2 + temp1) + 0.25 * invr * invr2 * log((r - sj) / (r + sj));
  }
  if (r > fabs(rho - sj)) {
    const double temp1 = 1.0 / (r + sj);
    const double invr3 = invr2 * invr;
    const double inv_rho = 1.0 / rho;
    return -0.25 * (-0.5 * (r2 - rho * rho + sj2) * invr3 * inv_rho * inv_rho +
                    invr * temp1 * (temp1 - invr) - invr3 * log(rho * temp1));
  }
  if (rho < sj) {
    const double temp1 = 1.0 / (r2 - sj2);
    return -0.5 * (sj * invr2 * temp1 - 2.0 * sj * temp1 * temp1 -
                   0.5 * invr2 * invr * log((sj - r) / (sj + r)));
  }
  return 0.0;
}

// ------------------------------------------------------------------------------------------------
// Pair functors for walkTile (lane l holds block I's atom, block J's atoms rotate)
// ------------------------------------------------------------------------------------------------
// Pass 1 payload: w1 = s * rho, w2 = rho, code = neck index
struct Radii64 {
  Stage64 v;
  Neck64 neck;
  double4 ai, bi;
  int ni;
  double psi_i, psi_j;
  __device__ Radii64(const Stage64 &v_in, const Neck64 &n) : v(v_in), neck(n) {}
  __device__ __forceinline__ void begin(int islot) {
    ai = v.pa[islot];
    bi = v.pb[islot];
    ni = v.code[islot];
    psi_i = psi_j = 0.0;
  }
  __device__ __forceinline__ void pair(int jslot, int) {
    const double4 aj = v.pa[jslot];
    const double4 bj = v.pb[jslot];
    const double dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    psi_i -= hctIntegral64(r, bi.x, aj.w);
    psi_j -= hctIntegral64(r, bj.x, ai.w);
    if (neck.size > 0 && r < bi.x + bj.x + neck.reach) {
      const int nj = v.code[jslot];
      double unused;
      psi_i -= neck.term(ni, nj, r, &unused);
      psi_j -= neck.term(nj, ni, r, &unused);
    }
  }
  __device__ __forceinline__ void rotate(int lane) {
    psi_j = __shfl_sync(0xffffffffu, psi_j, (lane + 1) & 31);
  }
};

// Pass 2 payload: w1 = charge x sqrt(Coulomb constant), w2 = effective radius
// Softened cores in FP64 (STORMM's Potential/soft_core_potentials.tpp, the FP32 path's
// softCorePair in double): the clash distance and sigma ratio of a system, scaled by its
// minimization progress when a cycle count is given
__device__ __forceinline__ double2 clashScaled64(const DevPrecise &p, int sysid) {
  const int cycle = (p.clash_cycle != nullptr) ? p.clash_cycle[sysid] : -1;
  if (cycle < 0) {
    return make_double2(p.clash_distance, p.clash_ratio);
  }
  if (cycle >= p.clash_cycles) {
    return make_double2(0.0, 0.0);
  }
  const double progress = static_cast<double>(p.clash_cycles - cycle) /
                          static_cast<double>(p.clash_cycles);
  return make_double2(p.clash_distance * progress, p.clash_ratio * progress);
}

template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH>
struct Pair64 {
  Stage64 v;
  const double2* lj;   // the molecule's Lennard-Jones table
  int nt;
  double kappa, inv_diel;
  double2 cl = make_double2(0.0, 0.0);   // the system's clash distance and sigma ratio
  double2 qc = make_double2(0.0, 0.0);   // its quadratic Coulomb core
  double4 ai, bi;
  int code_i;
  unsigned mask;
  double fxi, fyi, fzi, dei, fxj, fyj, fzj, dej;
  double e_elec, e_vdw, e_gb;
  __device__ Pair64(const Stage64 &v_in, const double2* lj_in, int nt_in, double kappa_in,
                    double inv_diel_in) :
      v(v_in), lj(lj_in), nt(nt_in), kappa(kappa_in), inv_diel(inv_diel_in) {}
  __device__ __forceinline__ void begin(int islot, unsigned mask_in) {
    ai = v.pa[islot];
    bi = v.pb[islot];
    code_i = v.code[islot] * nt;
    mask = mask_in;
    fxi = fyi = fzi = dei = fxj = fyj = fzj = dej = 0.0;
    e_elec = e_vdw = e_gb = 0.0;
  }
  __device__ __forceinline__ void pair(int jslot, int jl) {
    const double4 aj = v.pa[jslot];
    const double4 bj = v.pb[jslot];
    const double dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double qiqj = ai.w * aj.w;
    double fmag = 0.0;
    if (NB && CLASH && ((mask >> jl) & 1u) == 0u && (cl.x > 0.0 || cl.y > 0.0)) {
      const double invr = 1.0 / sqrt(r2);
      const double2 ab = lj[code_i + v.code[jslot]];
      double ee = 0.0, ev = 0.0;
      fmag = softCorePair64(r2 * invr, invr, qiqj, ab.x, ab.y, cl.x, qc, cl.y, &ee, &ev);
      if (ENERGY) {
        e_elec += ee;
        e_vdw += ev;
      }
      if (!FORCE) {
        fmag = 0.0;
      }
    }
    else if (NB && ((mask >> jl) & 1u) == 0u) {
      const double invr2 = 1.0 / r2;
      const double invr = sqrt(invr2);
      const double invr4 = invr2 * invr2;
      const double2 ab = lj[code_i + v.code[jslot]];
      if (ENERGY) {
        e_elec += qiqj * invr;
        e_vdw += (ab.x * invr4 * invr4 - ab.y * invr2) * invr4;
      }
      if (FORCE) {
        fmag = -(qiqj * invr * invr2) + (6.0 * ab.y - 12.0 * ab.x * invr4 * invr2) * invr4 * invr4;
      }
    }
    if (GB) {
      // nonbonded_potential.tpp:880-920
      const double ijb = bi.x * bj.x;
      const double efac = exp(-r2 / (4.0 * ijb));
      const double fgbi = 1.0 / sqrt(r2 + ijb * efac);
      const double fgbk = -kappa * kGbKscale64 / fgbi;
      const double expmkf = ((kappa > 0.0) ? exp(fgbk) : 1.0) * inv_diel;
      const double dielfac = 1.0 - expmkf;
      if (ENERGY) {
        e_gb -= qiqj * dielfac * fgbi;
      }
      if (FORCE) {
        const double temp6 = qiqj * fgbi * fgbi * fgbi * (dielfac + fgbk * expmkf);
        fmag += temp6 * (1.0 - 0.25 * efac);
        const double temp5 = 0.5 * efac * temp6 * (ijb + 0.25 * r2);
        dei += bi.x * temp5;
        dej += bj.x * temp5;
      }
    }
    if (FORCE) {
      fxi += fmag * dx;
      fyi += fmag * dy;
      fzi += fmag * dz;
      fxj -= fmag * dx;
      fyj -= fmag * dy;
      fzj -= fmag * dz;
    }
  }
  __device__ __forceinline__ void rotate(int lane) {
    if (FORCE) {
      const int src = (lane + 1) & 31;
      fxj = __shfl_sync(0xffffffffu, fxj, src);
      fyj = __shfl_sync(0xffffffffu, fyj, src);
      fzj = __shfl_sync(0xffffffffu, fzj, src);
      if (GB) {
        dej = __shfl_sync(0xffffffffu, dej, src);
      }
    }
  }
};

// Pass 3 payload: w1 = s * rho, w2 = rho, w3 = dE/dR after the chain-rule prefactor, code = neck
// index
struct Deriv64 {
  Stage64 v;
  Neck64 neck;
  double4 ai, bi;
  int ni;
  double fxi, fyi, fzi, fxj, fyj, fzj;
  __device__ Deriv64(const Stage64 &v_in, const Neck64 &n) : v(v_in), neck(n) {}
  __device__ __forceinline__ void begin(int islot) {
    ai = v.pa[islot];
    bi = v.pb[islot];
    ni = v.code[islot];
    fxi = fyi = fzi = fxj = fyj = fzj = 0.0;
  }
  __device__ __forceinline__ void pair(int jslot, int) {
    const double4 aj = v.pa[jslot];
    const double4 bj = v.pb[jslot];
    const double dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    double fmag = hctDerivative64(r, bi.x, aj.w) * bi.y + hctDerivative64(r, bj.x, ai.w) * bj.y;
    if (neck.size > 0 && r < bi.x + bj.x + neck.reach) {
      const int nj = v.code[jslot];
      double dij, dji;
      neck.term(ni, nj, r, &dij);
      neck.term(nj, ni, r, &dji);
      fmag += dij * bi.y + dji * bj.y;
    }
    fxi -= fmag * dx;
    fyi -= fmag * dy;
    fzi -= fmag * dz;
    fxj += fmag * dx;
    fyj += fmag * dy;
    fzj += fmag * dz;
  }
  __device__ __forceinline__ void rotate(int lane) {
    const int src = (lane + 1) & 31;
    fxj = __shfl_sync(0xffffffffu, fxj, src);
    fyj = __shfl_sync(0xffffffffu, fyj, src);
    fzj = __shfl_sync(0xffffffffu, fzj, src);
  }
};

// ------------------------------------------------------------------------------------------------
// Staging and the tile kernels
// ------------------------------------------------------------------------------------------------
// Stage a tile's atom blocks (block I in slots 0-31, block J in 32-63; a diagonal tile stages
// block I only).  Padding slots sit far apart with no charge, zero screened radius, a unit
// radius and zero dE/dR, so every term they enter vanishes for the real atom.
template <int PASS>
__device__ __forceinline__ void stageTile64(const DevSynthesis &d, const DevPrecise &p,
                                            const DevTiled &t, const Stage64 &v, int sysid,
                                            int I, int J, bool diag, int lane) {
  const int natom = d.atom_count[sysid];
  const int base = d.atom_start[sysid];
  for (int half = 0; half < (diag ? 1 : 2); half++) {
    const int a = (half == 0 ? I : J) * kTile + lane;
    const int slot = half * kTile + lane;
    double4 pa, pb;
    int code = 0;
    if (a < natom) {
      const int gi = base + a;
      pa = make_double4(static_cast<double>(d.xcrd[gi]) * d.inv_gpos_scale,
                        static_cast<double>(d.ycrd[gi]) * d.inv_gpos_scale,
                        static_cast<double>(d.zcrd[gi]) * d.inv_gpos_scale, 0.0);
      pb = make_double4(0.0, 0.0, 0.0, 0.0);
      code = (PASS == 2) ? d.lj_idx[gi] : ((d.neck_size > 0) ? d.neck_idx[gi] : 0);
      if (PASS == 2) {
        pa.w = p.charge[gi];
        pb.x = p.radius[gi];
      }
      else {
        pa.w = p.srho[gi];
        pb.x = p.rho[gi];
        if (PASS == 3) {
          pb.y = p.sde[gi];
        }
      }
    }
    else {
      pa = make_double4(5000.0 + 16.0 * static_cast<double>(slot), 0.0, 0.0, 0.0);
      pb = make_double4(1.0, 0.0, 0.0, 0.0);
    }
    v.pa[slot] = pa;
    v.pb[slot] = pb;
    v.code[slot] = code;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(256)
kRadii64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int tile_begin,
         int tile_end) {
  __shared__ double4 pa[kTiledWarps * kSlots64], pb[kTiledWarps * kSlots64];
  __shared__ int code[kTiledWarps * kSlots64];
  const int lane = threadIdx.x & 31;
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  const Stage64 v = warpStage(pa, pb, code);
  Radii64 f(v, Neck64(d, p));
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    stageTile64<1>(d, p, t, v, sysid, I, J, ti.diag, lane);
    f.begin(lane);
    walkTile(f, ti, lane);
    const int base = d.atom_start[sysid];
    if (lane < ti.ni) {
      addFixed(&t.psi_acc[base + I * kTile + lane], f.psi_i * kAcc64Scale);
    }
    const int jl = traveledAtom(ti, lane);
    if (jl < ti.nj) {
      addFixed(&t.psi_acc[base + J * kTile + jl], f.psi_j * kAcc64Scale);
    }
    __syncwarp();
  }
}

template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH>
__global__ void __launch_bounds__(256, 3)
kPair64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int tile_begin,
        int tile_end) {
  __shared__ double4 pa[kTiledWarps * kSlots64], pb[kTiledWarps * kSlots64];
  __shared__ int code[kTiledWarps * kSlots64];
  const int lane = threadIdx.x & 31;
  const double fs = static_cast<double>(d.frc_scale);
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  const Stage64 v = warpStage(pa, pb, code);
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    stageTile64<2>(d, p, t, v, sysid, I, J, ti.diag, lane);
    unsigned mask = 0u;
    if (NB) {
      const int midx = d.tile_mask_idx[d.tile_start[sysid] + ti.local];
      if (midx != 0) {
        mask = __ldg(&d.mask_pool[static_cast<size_t>(midx) * 32 + lane]);
      }
    }
    Pair64<FORCE, ENERGY, NB, GB, CLASH> f(v, p.ljab + d.lj_start[sysid], d.lj_ntypes[sysid],
                                           p.kappa, p.inv_dielectric);
    if (CLASH) {
      f.cl = clashScaled64(p, sysid);
      f.qc = quadraticCore64(f.cl.x);
    }
    f.begin(lane, mask);
    walkTile(f, ti, lane);
    const int base = d.atom_start[sysid];
    if (FORCE) {
      if (lane < ti.ni) {
        const int gi = base + I * kTile + lane;
        addFixed(&d.xfrc[gi], f.fxi * fs);
        addFixed(&d.yfrc[gi], f.fyi * fs);
        addFixed(&d.zfrc[gi], f.fzi * fs);
        if (GB) {
          addFixed(&t.de_acc[gi], f.dei * kAcc64Scale);
        }
      }
      const int jl = traveledAtom(ti, lane);
      if (jl < ti.nj) {
        const int gj = base + J * kTile + jl;
        addFixed(&d.xfrc[gj], f.fxj * fs);
        addFixed(&d.yfrc[gj], f.fyj * fs);
        addFixed(&d.zfrc[gj], f.fzj * fs);
        if (GB) {
          addFixed(&t.de_acc[gj], f.dej * kAcc64Scale);
        }
      }
    }
    if (ENERGY) {
      if (NB) {
        warpEnergy64(d, sysid, kElec, f.e_elec);
        warpEnergy64(d, sysid, kVdw, f.e_vdw);
      }
      if (GB) {
        warpEnergy64(d, sysid, kGb, f.e_gb);
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(256)
kDeriv64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int tile_begin,
         int tile_end) {
  __shared__ double4 pa[kTiledWarps * kSlots64], pb[kTiledWarps * kSlots64];
  __shared__ int code[kTiledWarps * kSlots64];
  const int lane = threadIdx.x & 31;
  const double fs = static_cast<double>(d.frc_scale);
  int first, last;
  warpTileRange(t, tile_begin, tile_end, &first, &last);
  const Stage64 v = warpStage(pa, pb, code);
  Deriv64 f(v, Neck64(d, p));
  for (int g = first; g < last; g++) {
    const int m = tiledOwner(t, g);
    const int sysid = t.systems[m];
    int I, J;
    const TileInfo ti = tiledTileInfo(d, sysid, g - t.tile_prefix[m], &I, &J);
    stageTile64<3>(d, p, t, v, sysid, I, J, ti.diag, lane);
    f.begin(lane);
    walkTile(f, ti, lane);
    const int base = d.atom_start[sysid];
    if (lane < ti.ni) {
      const int gi = base + I * kTile + lane;
      addFixed(&d.xfrc[gi], f.fxi * fs);
      addFixed(&d.yfrc[gi], f.fyi * fs);
      addFixed(&d.zfrc[gi], f.fzi * fs);
    }
    const int jl = traveledAtom(ti, lane);
    if (jl < ti.nj) {
      const int gj = base + J * kTile + jl;
      addFixed(&d.xfrc[gj], f.fxj * fs);
      addFixed(&d.yfrc[gj], f.fyj * fs);
      addFixed(&d.zfrc[gj], f.fzj * fs);
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------------------
// Per-atom steps between the pair passes (nonbonded_potential.tpp:730-805, 982-1021)
// ------------------------------------------------------------------------------------------------
template <bool FORCE, bool ENERGY, bool WS>
__global__ void __launch_bounds__(256)
kAtoms64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int atom_begin,
         int atom_end) {
  for (int q = atom_begin + blockIdx.x * blockDim.x + threadIdx.x; q < atom_end;
       q += gridDim.x * blockDim.x) {
    int sysid, a;
    const int gi = tiledAtom(d, t, q, &sysid, &a);
    double e_self = 0.0;
    double egbi = 1.0;
    if (a < d.atom_count[sysid]) {
      const double psi = static_cast<double>(t.psi_acc[gi]) * kInvAcc64Scale;
      const double rho = p.rho[gi];
      if (d.igb == SB_GB_HCT) {
        egbi = 1.0 / (1.0 / rho + psi);
        if (egbi < 0.0) {
          egbi = 30.0;
        }
      }
      else {
        const double fipsi = psi * (-rho);
        egbi = 1.0 / (1.0 / rho - tanh((p.alpha[gi] - p.beta[gi] * fipsi +
                                        p.gamma[gi] * fipsi * fipsi) * fipsi) / p.pb_radii[gi]);
      }
      const double qi = p.charge[gi];
      const double expmkf = ((p.kappa > 0.0) ? exp(-kGbKscale64 * p.kappa * egbi) : 1.0) *
                            p.inv_dielectric;
      const double atmq2h = 0.5 * qi * qi;
      const double atmqd2h = atmq2h * (1.0 - expmkf);
      e_self = -atmqd2h / egbi;
      if (FORCE) {
        addFixed(&t.de_acc[gi],
                 (atmqd2h - kGbKscale64 * p.kappa * atmq2h * expmkf * egbi) * kAcc64Scale);
      }
      if (WS) {
        d.born_radii[gi] = static_cast<float>(egbi);
        d.psi[gi] = __double2ll_rn(psi * d.psi_out_scale);
        d.psi_ovrf[gi] = 0;
      }
    }
    p.radius[gi] = egbi;
    if (ENERGY) {
      warpEnergy64(d, sysid, kGb, e_self);
    }
  }
}

template <bool WS>
__global__ void __launch_bounds__(256)
kChain64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int atom_begin,
         int atom_end) {
  for (int q = atom_begin + blockIdx.x * blockDim.x + threadIdx.x; q < atom_end;
       q += gridDim.x * blockDim.x) {
    int sysid, a;
    const int gi = tiledAtom(d, t, q, &sysid, &a);
    double sde = 0.0;
    if (a < d.atom_count[sysid]) {
      sde = static_cast<double>(t.de_acc[gi]) * kInvAcc64Scale;
      if (d.igb != SB_GB_HCT) {
        const double psi = static_cast<double>(t.psi_acc[gi]) * kInvAcc64Scale;
        const double rho = p.rho[gi];
        const double fipsi = psi * (-rho);
        const double al = p.alpha[gi], be = p.beta[gi], ga = p.gamma[gi];
        const double thi = tanh((al - (be - ga * fipsi) * fipsi) * fipsi);
        sde *= (al - (2.0 * be - 3.0 * ga * fipsi) * fipsi) * (1.0 - thi * thi) * rho /
               p.pb_radii[gi];
      }
      if (WS) {
        d.sumdeijda[gi] = __double2ll_rn(sde * d.psi_out_scale);
        d.sumdeijda_ovrf[gi] = 0;
      }
    }
    p.sde[gi] = sde;
  }
}

// ------------------------------------------------------------------------------------------------
// Valence terms, one thread per term (the oracle-style restatement of valence_potential.tpp)
// ------------------------------------------------------------------------------------------------
// System owning term index k of a system-major term list with prefix `start` (nsys + 1)
__device__ __forceinline__ int termOwner(const int* start, int nsys, int k) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= k) {
      lo = mid;
    }
    else {
      hi = mid - 1;
    }
  }
  return lo;
}

struct Atoms64 {
  const DevSynthesis &d;
  int base;
  __device__ __forceinline__ double3 at(int a) const {
    const int gi = base + a;
    return make_double3(static_cast<double>(d.xcrd[gi]) * d.inv_gpos_scale,
                        static_cast<double>(d.ycrd[gi]) * d.inv_gpos_scale,
                        static_cast<double>(d.zcrd[gi]) * d.inv_gpos_scale);
  }
  __device__ __forceinline__ void force(int a, double fx, double fy, double fz) const {
    const double fs = static_cast<double>(d.frc_scale);
    addFixed(&d.xfrc[base + a], fx * fs);
    addFixed(&d.yfrc[base + a], fy * fs);
    addFixed(&d.zfrc[base + a], fz * fs);
  }
};

__device__ __forceinline__ double3 sub3(double3 a, double3 b) {
  return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double dot3(double3 a, double3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ void energyAdd(const DevSynthesis &d, int sysid, int slot, double e) {
  const long long v = __double2ll_rn(e * static_cast<double>(d.nrg_scale));
  if (v != 0) {
    atomicAdd(&d.energies[static_cast<size_t>(sysid) * kNrgStride + slot],
              static_cast<unsigned long long>(v));
  }
}

// Terms of the systems of tiled molecules [mol_begin, mol_end): the FP64 mode routes every
// system to the tiled path in system order, so those molecules are consecutive systems
template <bool FORCE, bool ENERGY, bool CLASH>
__global__ void __launch_bounds__(256)
kValence64(const DevSynthesis d, const DevPrecise p, const DevTiled t, int mol_begin,
           int mol_end) {
  const int stride = gridDim.x * blockDim.x;
  const int first_sys = t.systems[mol_begin];
  const int last_sys = t.systems[mol_end - 1];
  // harmonic bonds, valence_potential.tpp:9-97
  for (int k = d.bond_start[first_sys] + blockIdx.x * blockDim.x + threadIdx.x;
       k < d.bond_start[last_sys + 1]; k += stride) {
    const int sysid = termOwner(d.bond_start, d.nsys, k);
    const Atoms64 at{d, d.atom_start[sysid]};
    const int2 ij = p.bond_atoms[k];
    const double2 kr = p.bond_prm[k];
    const double3 dv = sub3(at.at(ij.y), at.at(ij.x));
    const double r = sqrt(dot3(dv, dv));
    const double dl = r - kr.y;
    if (FORCE) {
      const double fmag = 2.0 * kr.x * dl / r;
      at.force(ij.x, fmag * dv.x, fmag * dv.y, fmag * dv.z);
      at.force(ij.y, -fmag * dv.x, -fmag * dv.y, -fmag * dv.z);
    }
    if (ENERGY) {
      energyAdd(d, sysid, kBond, kr.x * dl * dl);
    }
  }
  // harmonic angles, valence_potential.tpp:170-288
  for (int k = d.angl_start[first_sys] + blockIdx.x * blockDim.x + threadIdx.x;
       k < d.angl_start[last_sys + 1]; k += stride) {
    const int sysid = termOwner(d.angl_start, d.nsys, k);
    const Atoms64 at{d, d.atom_start[sysid]};
    const int4 ijk = p.angl_atoms[k];
    const double2 kt = p.angl_prm[k];
    const double3 cj = at.at(ijk.y);
    const double3 ba = sub3(at.at(ijk.x), cj);
    const double3 bc = sub3(at.at(ijk.z), cj);
    const double mgba = dot3(ba, ba);
    const double mgbc = dot3(bc, bc);
    const double invbabc = 1.0 / sqrt(mgba * mgbc);
    const double costheta = fmin(1.0, fmax(-1.0, dot3(ba, bc) * invbabc));
    const double dtheta = acos(costheta) - kt.y;
    if (FORCE) {
      const double dA = -2.0 * kt.x * dtheta / sqrt(1.0 - costheta * costheta);
      const double sqba = dA / mgba;
      const double sqbc = dA / mgbc;
      const double mbabc = dA * invbabc;
      const double3 adf = make_double3(bc.x * mbabc - costheta * ba.x * sqba,
                                       bc.y * mbabc - costheta * ba.y * sqba,
                                       bc.z * mbabc - costheta * ba.z * sqba);
      const double3 cdf = make_double3(ba.x * mbabc - costheta * bc.x * sqbc,
                                       ba.y * mbabc - costheta * bc.y * sqbc,
                                       ba.z * mbabc - costheta * bc.z * sqbc);
      at.force(ijk.x, -adf.x, -adf.y, -adf.z);
      at.force(ijk.y, adf.x + cdf.x, adf.y + cdf.y, adf.z + cdf.z);
      at.force(ijk.z, -cdf.x, -cdf.y, -cdf.z);
    }
    if (ENERGY) {
      energyAdd(d, sysid, kAngle, kt.x * dtheta * dtheta);
    }
  }
  // cosine dihedrals with attached 1-4 pairs, valence_potential.tpp:359-578, 1288-1420
  for (int k = d.dihe_start[first_sys] + blockIdx.x * blockDim.x + threadIdx.x;
       k < d.dihe_start[last_sys + 1]; k += stride) {
    const int sysid = termOwner(d.dihe_start, d.nsys, k);
    const Atoms64 at{d, d.atom_start[sysid]};
    const int4 ijkl = p.dihe_atoms[k];
    const double4 prm = p.dihe_prm[k];     // amplitude, periodicity, phase, improper flag
    const double2 attn = p.dihe_attn[k];   // 1 / scee, 1 / scnb (0: no 1-4 pair)
    const double3 ci = at.at(ijkl.x), cj = at.at(ijkl.y), ck = at.at(ijkl.z);
    const double3 cl = at.at(ijkl.w);
    const double3 ab = sub3(cj, ci), bc = sub3(ck, cj), cd = sub3(cl, ck);
    double3 crabbc = cross3(ab, bc);
    double3 crbccd = cross3(bc, cd);
    double costheta = dot3(crabbc, crbccd) / sqrt(dot3(crabbc, crabbc) * dot3(crbccd, crbccd));
    costheta = fmin(1.0, fmax(-1.0, costheta));
    const double3 scr = cross3(crabbc, crbccd);
    const double sgn = (dot3(scr, bc) > 0.0) ? 1.0 : -1.0;
    double theta;
    if (fabs(costheta) >= kNearToOne) {
      // Math/rounding.tpp:25-60: the arcsine route near 0 and pi
      const double ia = 1.0 / sqrt(dot3(crabbc, crabbc));
      const double ib = 1.0 / sqrt(dot3(crbccd, crbccd));
      double3 rd = make_double3(crbccd.x * ib - crabbc.x * ia, crbccd.y * ib - crabbc.y * ia,
                                crbccd.z * ib - crabbc.z * ia);
      double rs = sqrt(dot3(rd, rd));
      if (fabs(rs) > 1.0) {
        rd = make_double3(crbccd.x * ib + crabbc.x * ia, crbccd.y * ib + crabbc.y * ia,
                          crbccd.z * ib + crabbc.z * ia);
        rs = kPi64 - sqrt(dot3(rd, rd));
      }
      theta = sgn * rs;
    }
    else {
      theta = sgn * acos(costheta);
    }
    const double sangle = prm.y * theta - prm.z;
    if (FORCE) {
      const double fr = prm.x * prm.y * sin(sangle);
      const double mgab = sqrt(dot3(ab, ab));
      const double mgbc = sqrt(dot3(bc, bc));
      const double mgcd = sqrt(dot3(cd, cd));
      const double invab = 1.0 / mgab, invbc = 1.0 / mgbc, invcd = 1.0 / mgcd;
      const double cosb = -dot3(ab, bc) * invab * invbc;
      const double cosc = -dot3(bc, cd) * invbc * invcd;
      const double isinb2 = (cosb * cosb < kAsymptoticToOne) ? fr / (1.0 - cosb * cosb) :
                                                                fr * kInvOneMinusAsymptote;
      const double isinc2 = (cosc * cosc < kAsymptoticToOne) ? fr / (1.0 - cosc * cosc) :
                                                                fr * kInvOneMinusAsymptote;
      const double invabc = invab * invbc, invbcd = invbc * invcd;
      crabbc = make_double3(crabbc.x * invabc, crabbc.y * invabc, crabbc.z * invabc);
      crbccd = make_double3(crbccd.x * invbcd, crbccd.y * invbcd, crbccd.z * invbcd);
      const double fa = -invab * isinb2;
      const double fb1 = (mgbc - mgab * cosb) * invabc * isinb2;
      const double fb2 = cosc * invbc * isinc2;
      const double fd = -invcd * isinc2;
      const double3 fi = make_double3(crabbc.x * fa, crabbc.y * fa, crabbc.z * fa);
      const double3 fj = make_double3(fb1 * crabbc.x - fb2 * crbccd.x,
                                      fb1 * crabbc.y - fb2 * crbccd.y,
                                      fb1 * crabbc.z - fb2 * crbccd.z);
      const double3 fl = make_double3(-fd * crbccd.x, -fd * crbccd.y, -fd * crbccd.z);
      at.force(ijkl.x, fi.x, fi.y, fi.z);
      at.force(ijkl.y, fj.x, fj.y, fj.z);
      at.force(ijkl.z, -(fi.x + fj.x + fl.x), -(fi.y + fj.y + fl.y), -(fi.z + fj.z + fl.z));
      at.force(ijkl.w, fl.x, fl.y, fl.z);
    }
    if (ENERGY) {
      energyAdd(d, sysid, (prm.w != 0.0) ? kImproperDihedral : kProperDihedral,
                prm.x * (1.0 + cos(sangle)));
    }
    if (attn.x > 0.0) {
      const double3 dv = sub3(cl, ci);
      const int gi = d.atom_start[sysid] + ijkl.x;
      const int gl = d.atom_start[sysid] + ijkl.w;
      const int nt = d.lj_ntypes[sysid];
      const double2 ab14 = p.ljab14[d.lj_start[sysid] + d.lj_idx[gi] * nt + d.lj_idx[gl]];
      const double lja = ab14.x * attn.y;
      const double ljb = ab14.y * attn.y;
      const double qiqj = p.charge[gi] * p.charge[gl] * attn.x;
      const double invr2 = 1.0 / dot3(dv, dv);
      const double invr = sqrt(invr2);
      const double invr4 = invr2 * invr2;
      const double2 cl = CLASH ? clashScaled64(p, sysid) : make_double2(0.0, 0.0);
      if (CLASH && (cl.x > 0.0 || cl.y > 0.0)) {
        // clash-softened 1-4 pair (valence_potential.tpp:1337-1357)
        double ee = 0.0, ev = 0.0;
        const double fmag = softCorePair64(1.0 / invr, invr, qiqj, lja, ljb, cl.x,
                                           quadraticCore64(cl.x), cl.y, &ee, &ev);
        if (FORCE) {
          at.force(ijkl.x, fmag * dv.x, fmag * dv.y, fmag * dv.z);
          at.force(ijkl.w, -fmag * dv.x, -fmag * dv.y, -fmag * dv.z);
        }
        if (ENERGY) {
          energyAdd(d, sysid, kElec14, ee);
          energyAdd(d, sysid, kVdw14, ev);
        }
      }
      else {
        if (FORCE) {
          const double fmag = -(qiqj * invr * invr2) +
                              (6.0 * ljb - 12.0 * lja * invr4 * invr2) * invr4 * invr4;
          at.force(ijkl.x, fmag * dv.x, fmag * dv.y, fmag * dv.z);
          at.force(ijkl.w, -fmag * dv.x, -fmag * dv.y, -fmag * dv.z);
        }
        if (ENERGY) {
          energyAdd(d, sysid, kElec14, qiqj * invr);
          energyAdd(d, sysid, kVdw14, lja * invr4 * invr4 * invr4 - ljb * invr4 * invr2);
        }
      }
    }
  }
}

}  // namespace

// All requested terms of tiled molecules [mol_begin, mol_end) in FP64.  psi_acc and de_acc of
// those molecules' atoms must be zero on entry (the caller clears them on the stream).
cudaError_t launchTiled64(const DevSynthesis &d, const DevPrecise &p, const DevTiled &t,
                          const int* h_tile_prefix, const int* h_atom_prefix, int mol_begin,
                          int mol_end, int terms, bool force, bool energy, bool workspace,
                          int sm_count, cudaStream_t stream, bool clash) {
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
  if (vale) {
    const int vgrid = sm_count * 4;
#define SB_VALE64(C)                                                                            \
    if (force && energy) kValence64<true, true, C><<<vgrid, 256, 0, stream>>>(d, p, t, mol_begin, mol_end); \
    else if (force) kValence64<true, false, C><<<vgrid, 256, 0, stream>>>(d, p, t, mol_begin, mol_end);    \
    else kValence64<false, true, C><<<vgrid, 256, 0, stream>>>(d, p, t, mol_begin, mol_end);
    if (clash) { SB_VALE64(true) }
    else { SB_VALE64(false) }
#undef SB_VALE64
  }
  if (gb) {
    kRadii64<<<tgrid, 256, 0, stream>>>(d, p, t, tb, te);
#define SB_ATOMS(F, E) \
    if (workspace) kAtoms64<F, E, true><<<agrid, 256, 0, stream>>>(d, p, t, ab, ae); \
    else kAtoms64<F, E, false><<<agrid, 256, 0, stream>>>(d, p, t, ab, ae);
    if (force && energy) { SB_ATOMS(true, true) }
    else if (force) { SB_ATOMS(true, false) }
    else { SB_ATOMS(false, true) }
#undef SB_ATOMS
  }
  if (nb || gb) {
#define SB_PAIR(F, E)                                                                       \
    if (nb && gb && clash) kPair64<F, E, true, true, true><<<tgrid, 256, 0, stream>>>(d, p, t, tb, te); \
    else if (nb && gb) kPair64<F, E, true, true, false><<<tgrid, 256, 0, stream>>>(d, p, t, tb, te);    \
    else if (nb && clash) kPair64<F, E, true, false, true><<<tgrid, 256, 0, stream>>>(d, p, t, tb, te); \
    else if (nb) kPair64<F, E, true, false, false><<<tgrid, 256, 0, stream>>>(d, p, t, tb, te);         \
    else kPair64<F, E, false, true, false><<<tgrid, 256, 0, stream>>>(d, p, t, tb, te);
    if (force && energy) { SB_PAIR(true, true) }
    else if (force) { SB_PAIR(true, false) }
    else { SB_PAIR(false, true) }
#undef SB_PAIR
  }
  if (gb && force) {
    if (workspace) kChain64<true><<<agrid, 256, 0, stream>>>(d, p, t, ab, ae);
    else kChain64<false><<<agrid, 256, 0, stream>>>(d, p, t, ab, ae);
    kDeriv64<<<tgrid, 256, 0, stream>>>(d, p, t, tb, te);
  }
  return cudaGetLastError();
}

}  // namespace sb
