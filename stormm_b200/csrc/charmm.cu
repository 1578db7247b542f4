// CHARMM terms and restraints of a synthesis, in FP64 from the exact fixed-point coordinates,
// one thread per term, after the fused pass (or the tiled / FP64 path) has evaluated everything
// else:
//
//   Urey-Bradley     k (r_ik - r0)^2 between the outer atoms of an angle
//                    (Potential/valence_potential.tpp:659-691 with evalHarmonicStretch)
//   CHARMM improper  k (theta - phase)^2, theta the signed dihedral angle of atoms i-j-k-l,
//                    no periodic wrap of theta - phase (valence_potential.tpp:722-760 with
//                    evalDihedralTwist, DihedralStyle::HARMONIC)
//   CMAP             a bicubic spline over (phi, psi), the dihedrals of atoms 0-3 and 1-4, each
//                    shifted by pi into [0, 2 pi) and mapped onto the surface's grid cells
//                    (valence_potential.tpp:789-1222); the 16 coefficients of each cell are
//                    built on the host (cmapPatches in synthesis.cu)
//   restraints       STORMM's flat-bottom positional, distance, angle and dihedral restraints
//                    (valence_potential.tpp:1558-2050), constant ones
//
// Every force and energy enters the int64 accumulators through integer atomics of the term's
// own contribution rounded to the fixed-point grid, so sums do not depend on scheduling; the
// energy of each term is rounded as STORMM's ScoreCard rounds it (llround of the term times
// 2^nrg_bits).
#include <cuda_runtime.h>

#include "device_kits.h"
#include "unit_eval.cuh"

namespace sb {

namespace {

constexpr int kSlotUreyBradley = 4;      // StateVariable::UREY_BRADLEY
constexpr int kSlotCharmmImproper = 5;   // StateVariable::CHARMM_IMPROPER
constexpr int kSlotCmap = 6;             // StateVariable::CMAP
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kPi = 3.1415926535897932384626433832795;

__device__ __forceinline__ double3 displacement(const DevCharmm &c, int from, int to) {
  return make_double3(static_cast<double>(c.xcrd[to] - c.xcrd[from]) * c.inv_gpos_scale,
                      static_cast<double>(c.ycrd[to] - c.ycrd[from]) * c.inv_gpos_scale,
                      static_cast<double>(c.zcrd[to] - c.zcrd[from]) * c.inv_gpos_scale);
}

__device__ __forceinline__ void addForce(const DevCharmm &c, int atom, double fx, double fy,
                                         double fz) {
  atomicAdd(reinterpret_cast<unsigned long long*>(&c.xfrc[atom]),
            static_cast<unsigned long long>(__double2ll_rn(fx * c.frc_scale)));
  atomicAdd(reinterpret_cast<unsigned long long*>(&c.yfrc[atom]),
            static_cast<unsigned long long>(__double2ll_rn(fy * c.frc_scale)));
  atomicAdd(reinterpret_cast<unsigned long long*>(&c.zfrc[atom]),
            static_cast<unsigned long long>(__double2ll_rn(fz * c.frc_scale)));
}

__device__ __forceinline__ void addEnergy(const DevCharmm &c, int sys, int slot, double e) {
  atomicAdd(&c.energies[static_cast<size_t>(sys) * kNrgStride + slot],
            static_cast<unsigned long long>(__double2ll_rn(e * c.nrg_scale)));
}

// The signed dihedral angle of ab, bc, cd (positive when (ab x bc) x (bc x cd) points along bc),
// from atan2, well conditioned near 0 and pi
__device__ __forceinline__ double dihedralAngle(double3 ab, double3 bc, double3 cd) {
  const double3 n1 = cross3d(ab, bc);
  const double3 n2 = cross3d(bc, cd);
  return atan2(sqrt(dot3d(bc, bc)) * dot3d(ab, n2), dot3d(n1, n2));
}

// Forces of a dihedral term on its four atoms given g = -dE/dtheta: the gradient of the angle
// in the form STORMM applies it (valence_potential.tpp:456-500), the third atom taking minus
// the sum of the others
__device__ void dihedralForces(const DevCharmm &c, int ia, int ja, int ka, int la, double3 ab,
                               double3 bc, double3 cd, double g) {
  const double ab2 = dot3d(ab, ab), bc2 = dot3d(bc, bc), cd2 = dot3d(cd, cd);
  const double invab = rsqrt(ab2), invbc = rsqrt(bc2), invcd = rsqrt(cd2);
  const double mgab = ab2 * invab, mgbc = bc2 * invbc;
  const double cosb = -dot3d(ab, bc) * invab * invbc;
  const double cosc = -dot3d(bc, cd) * invbc * invcd;
  const double isinb2 = (cosb * cosb < kAsymptoticToOne) ? g / (1.0 - cosb * cosb)
                                                         : g * kInvOneMinusAsymptote;
  const double isinc2 = (cosc * cosc < kAsymptoticToOne) ? g / (1.0 - cosc * cosc)
                                                         : g * kInvOneMinusAsymptote;
  const double invabc = invab * invbc, invbcd = invbc * invcd;
  double3 n1 = cross3d(ab, bc), n2 = cross3d(bc, cd);
  n1 = make_double3(n1.x * invabc, n1.y * invabc, n1.z * invabc);
  n2 = make_double3(n2.x * invbcd, n2.y * invbcd, n2.z * invbcd);
  const double fa = -invab * isinb2;
  const double fb1 = (mgbc - mgab * cosb) * invabc * isinb2;
  const double fb2 = cosc * invbc * isinc2;
  const double fd = -invcd * isinc2;
  const double3 fi = make_double3(n1.x * fa, n1.y * fa, n1.z * fa);
  const double3 fj = make_double3(fb1 * n1.x - fb2 * n2.x, fb1 * n1.y - fb2 * n2.y,
                                  fb1 * n1.z - fb2 * n2.z);
  const double3 fl = make_double3(-fd * n2.x, -fd * n2.y, -fd * n2.z);
  addForce(c, ia, fi.x, fi.y, fi.z);
  addForce(c, ja, fj.x, fj.y, fj.z);
  addForce(c, ka, -(fi.x + fj.x + fl.x), -(fi.y + fj.y + fl.y), -(fi.z + fj.z + fl.z));
  addForce(c, la, fl.x, fl.y, fl.z);
}

// A dihedral shifted by pi into [0, 2 pi), as the CMAP grid indexes it
__device__ __forceinline__ double cmapAngle(double theta) {
  double a = theta + kPi;
  a = (a < 0.0) ? a + kTwoPi : ((a >= kTwoPi) ? a - kTwoPi : a);
  return a;
}

template <bool FORCE, bool ENERGY>
__global__ void __launch_bounds__(128)
kCharmmTerms(const DevCharmm c, int ub0, int nub, int ci0, int nci, int cm0, int ncm) {
  const int total = nub + nci + ncm;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    if (t < nub) {
      const int4 u = c.ubrd[ub0 + t];
      const double2 p = c.ubrd_prm[ub0 + t];
      const double3 d = displacement(c, u.x, u.y);
      const double r = sqrt(dot3d(d, d));
      const double dr = r - p.y;
      if (ENERGY) addEnergy(c, u.z, kSlotUreyBradley, p.x * dr * dr);
      if (FORCE) {
        // force on atom k: -dE/dr along the bond, atom i the opposite
        const double f = -2.0 * p.x * dr / r;
        addForce(c, u.y, f * d.x, f * d.y, f * d.z);
        addForce(c, u.x, -f * d.x, -f * d.y, -f * d.z);
      }
      continue;
    }
    if (t < nub + nci) {
      const int k = ci0 + t - nub;
      const int4 a = c.cimp[k];
      const double2 p = c.cimp_prm[k];
      const double3 ab = displacement(c, a.x, a.y);
      const double3 bc = displacement(c, a.y, a.z);
      const double3 cd = displacement(c, a.z, a.w);
      const double s = dihedralAngle(ab, bc, cd) - p.y;
      if (ENERGY) addEnergy(c, c.cimp_sys[k], kSlotCharmmImproper, p.x * s * s);
      if (FORCE) dihedralForces(c, a.x, a.y, a.z, a.w, ab, bc, cd, -2.0 * p.x * s);
      continue;
    }
    const int k = cm0 + t - nub - nci;
    const int4 a = c.cmap[k];
    const int4 b = c.cmap_b[k];
    const int2 surf = c.cmap_surf[b.z];
    const double3 ab = displacement(c, a.x, a.y);
    const double3 bc = displacement(c, a.y, a.z);
    const double3 cd = displacement(c, a.z, a.w);
    const double3 de = displacement(c, a.w, b.x);
    const double dim = static_cast<double>(surf.y);
    const double phi_grid = cmapAngle(dihedralAngle(ab, bc, cd)) * dim / kTwoPi;
    const double psi_grid = cmapAngle(dihedralAngle(bc, cd, de)) * dim / kTwoPi;
    const int iphi = max(0, min(static_cast<int>(phi_grid), surf.y - 1));
    const int ipsi = max(0, min(static_cast<int>(psi_grid), surf.y - 1));
    const double u = phi_grid - iphi;
    const double v = psi_grid - ipsi;
    // coefficient a[r + 4 s] multiplies u^r v^s
    const double* acoef = c.cmap_patch + (static_cast<size_t>(surf.x) +
                                          static_cast<size_t>(ipsi) * surf.y + iphi) * 16;
    double e = 0.0, de_du = 0.0, de_dv = 0.0;
    for (int r = 3; r >= 0; r--) {
      // row polynomial in v and its derivative, then Horner in u
      const double q = ((acoef[r + 12] * v + acoef[r + 8]) * v + acoef[r + 4]) * v + acoef[r];
      const double dq = (3.0 * acoef[r + 12] * v + 2.0 * acoef[r + 8]) * v + acoef[r + 4];
      de_du = de_du * u + e;
      e = e * u + q;
      de_dv = de_dv * u + dq;
    }
    if (ENERGY) addEnergy(c, b.y, kSlotCmap, e);
    if (FORCE) {
      const double scale = dim / kTwoPi;   // grid units per radian
      dihedralForces(c, a.x, a.y, a.z, a.w, ab, bc, cd, -de_du * scale);
      dihedralForces(c, a.y, a.z, a.w, b.x, bc, cd, de, -de_dv * scale);
    }
  }
}

constexpr int kSlotRestraint = 12;       // StateVariable::RESTRAINT

// The flat-bottom potential of a restrained value d (Restraints/restraint_util.tpp:9-46):
// returns the energy and sets *g = -dE/dd
__device__ __forceinline__ double flatBottom(double d, double2 k, double4 r, double* g) {
  double keq, dl, e;
  if (d < r.x) {
    dl = r.x - r.y;
    keq = k.x;
    e = keq * (dl * dl + 2.0 * dl * (d - r.x));
  }
  else if (d < r.y) {
    dl = d - r.y;
    keq = k.x;
    e = keq * dl * dl;
  }
  else if (d < r.z) {
    dl = 0.0;
    keq = 0.0;
    e = 0.0;
  }
  else if (d < r.w) {
    dl = d - r.z;
    keq = k.y;
    e = keq * dl * dl;
  }
  else {
    dl = r.w - r.z;
    keq = k.y;
    e = keq * (dl * dl + 2.0 * dl * (d - r.w));
  }
  *g = -2.0 * keq * dl;
  return e;
}

// Weights of the initial and final values at a step (Restraints/restraint_util.tpp:48-75)
__device__ __forceinline__ double2 restraintMixture(int step, int2 s) {
  if (step < s.x) return make_double2(0.0, 0.0);
  if (s.x == s.y) return make_double2(1.0, 0.0);
  if (step < s.y) {
    const double w = static_cast<double>(step - s.x) / static_cast<double>(s.y - s.x);
    return make_double2(1.0 - w, w);
  }
  return make_double2(0.0, 1.0);
}

// w.x a + w.y b, each product rounded before the sum as the host code rounds it
__device__ __forceinline__ double mix(double2 w, double a, double b) {
  return __dadd_rn(__dmul_rn(w.x, a), __dmul_rn(w.y, b));
}

template <bool FORCE, bool ENERGY>
__global__ void __launch_bounds__(128)
kRestraints(const DevCharmm c, int first, int count) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    const int q = first + t;
    const int4 a = c.rst_atoms[q];
    const int2 meta = c.rst_meta[q];
    const int step = (c.rst_cycle != nullptr) ? c.rst_cycle[meta.y] : c.rst_step;
    const double2 w = restraintMixture(step, c.rst_steps[q]);
    const double2 k0 = c.rst_k[q], k1 = c.rst_kf[q];
    const double4 r0 = c.rst_r[q], r1 = c.rst_rf[q];
    const double2 k = make_double2(mix(w, k0.x, k1.x), mix(w, k0.y, k1.y));
    const double4 r = make_double4(mix(w, r0.x, r1.x), mix(w, r0.y, r1.y), mix(w, r0.z, r1.z),
                                   mix(w, r0.w, r1.w));
    double e = 0.0, g = 0.0;
    if (meta.x == 1) {
      // positional: distance of the atom from the target point
      const double4 t0 = c.rst_target[q], t1 = c.rst_target_f[q];
      const double3 tg = make_double3(mix(w, t0.x, t1.x), mix(w, t0.y, t1.y),
                                      mix(w, t0.z, t1.z));
      const double3 d = make_double3(static_cast<double>(c.xcrd[a.x]) * c.inv_gpos_scale - tg.x,
                                     static_cast<double>(c.ycrd[a.x]) * c.inv_gpos_scale - tg.y,
                                     static_cast<double>(c.zcrd[a.x]) * c.inv_gpos_scale - tg.z);
      const double dr = sqrt(dot3d(d, d));
      e = flatBottom(dr, k, r, &g);
      if (FORCE) {
        if (dr < 1.0e-8) {
          // at the target itself the direction is arbitrary: the force is split evenly over
          // the three axes, as the reference does
          const double f = g / sqrt(3.0);
          addForce(c, a.x, f, f, f);
        }
        else {
          const double f = g / dr;
          addForce(c, a.x, f * d.x, f * d.y, f * d.z);
        }
      }
    }
    else if (meta.x == 2) {
      const double3 d = displacement(c, a.x, a.y);
      const double dr = sqrt(dot3d(d, d));
      e = flatBottom(dr, k, r, &g);
      if (FORCE) {
        const double f = g / dr;
        addForce(c, a.y, f * d.x, f * d.y, f * d.z);
        addForce(c, a.x, -f * d.x, -f * d.y, -f * d.z);
      }
    }
    else if (meta.x == 3) {
      // angle at the second atom, from acos of the normalized dot product as the reference
      // measures it
      const double3 ba = displacement(c, a.y, a.x);
      const double3 bc = displacement(c, a.y, a.z);
      const double inv_ba = rsqrt(dot3d(ba, ba)), inv_bc = rsqrt(dot3d(bc, bc));
      double cs = dot3d(ba, bc) * inv_ba * inv_bc;
      cs = fmin(1.0, fmax(-1.0, cs));
      e = flatBottom(acos(cs), k, r, &g);
      if (FORCE) {
        // dtheta/dr_i = -(bc / (|ba||bc|) - cos ba / |ba|^2) / sin
        const double s = g / sqrt(fmax(1.0 - cs * cs, 1.0e-30));
        const double3 fi = make_double3(-s * (bc.x * inv_ba * inv_bc - cs * ba.x * inv_ba * inv_ba),
                                        -s * (bc.y * inv_ba * inv_bc - cs * ba.y * inv_ba * inv_ba),
                                        -s * (bc.z * inv_ba * inv_bc - cs * ba.z * inv_ba * inv_ba));
        const double3 fk = make_double3(-s * (ba.x * inv_ba * inv_bc - cs * bc.x * inv_bc * inv_bc),
                                        -s * (ba.y * inv_ba * inv_bc - cs * bc.y * inv_bc * inv_bc),
                                        -s * (ba.z * inv_ba * inv_bc - cs * bc.z * inv_bc * inv_bc));
        addForce(c, a.x, fi.x, fi.y, fi.z);
        addForce(c, a.z, fk.x, fk.y, fk.z);
        addForce(c, a.y, -(fi.x + fk.x), -(fi.y + fk.y), -(fi.z + fk.z));
      }
    }
    else {
      const double3 ab = displacement(c, a.x, a.y);
      const double3 bc = displacement(c, a.y, a.z);
      const double3 cd = displacement(c, a.z, a.w);
      // the midpoint mixes the end points' sums (valence_potential.tpp:1954)
      const double mid = 0.5 * mix(w, r0.y + r0.z, r1.y + r1.z);
      double th = dihedralAngle(ab, bc, cd) - mid;
      th -= kTwoPi * rint(th / kTwoPi);       // within pi of the midpoint
      e = flatBottom(mid + th, k, r, &g);
      if (FORCE) dihedralForces(c, a.x, a.y, a.z, a.w, ab, bc, cd, g);
    }
    if (ENERGY) addEnergy(c, meta.y, kSlotRestraint, e);
  }
}

}  // namespace

cudaError_t launchRestraints(const DevCharmm &c, int first, int count, bool force, bool energy,
                             int sm_count, cudaStream_t stream) {
  if (count == 0 || (!force && !energy)) return cudaSuccess;
  int blocks = (count + 127) / 128;
  const int cap = 8 * (sm_count > 0 ? sm_count : 148);
  blocks = blocks > cap ? cap : blocks;
  if (force && energy) {
    kRestraints<true, true><<<blocks, 128, 0, stream>>>(c, first, count);
  }
  else if (force) {
    kRestraints<true, false><<<blocks, 128, 0, stream>>>(c, first, count);
  }
  else {
    kRestraints<false, true><<<blocks, 128, 0, stream>>>(c, first, count);
  }
  return cudaGetLastError();
}

cudaError_t launchCharmmTerms(const DevCharmm &c, int ub0, int nub, int ci0, int nci, int cm0,
                              int ncm, bool force, bool energy, int sm_count,
                              cudaStream_t stream) {
  const int total = nub + nci + ncm;
  if (total == 0 || (!force && !energy)) return cudaSuccess;
  int blocks = (total + 127) / 128;
  const int cap = 8 * (sm_count > 0 ? sm_count : 148);
  blocks = blocks > cap ? cap : blocks;
  if (force && energy) {
    kCharmmTerms<true, true><<<blocks, 128, 0, stream>>>(c, ub0, nub, ci0, nci, cm0, ncm);
  }
  else if (force) {
    kCharmmTerms<true, false><<<blocks, 128, 0, stream>>>(c, ub0, nub, ci0, nci, cm0, ncm);
  }
  else {
    kCharmmTerms<false, true><<<blocks, 128, 0, stream>>>(c, ub0, nub, ci0, nci, cm0, ncm);
  }
  return cudaGetLastError();
}

}  // namespace sb
