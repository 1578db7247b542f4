// Device building blocks of the fused batched evaluation of valence, Coulomb + Lennard-Jones and
// Generalized Born terms, shared by the evaluation kernel and the minimization kernel.
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
//               sums (nonbonded_potential.tpp:8-425, 808-975)
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
// per-atom values, gbv the reciprocal effective radius with the Lennard-Jones code (pass 2) and
// then the chain-rule dE/dR (pass 3).
#ifndef STORMM_B200_UNIT_EVAL_CUH
#define STORMM_B200_UNIT_EVAL_CUH

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "device_kits.h"
#include "fixed_point.cuh"

namespace sb {

namespace {

// Constants/generalized_born.h:21-44 (Taylor series of the HCT integral at long range)
constexpr float kTaylorA = 0.33333333333333333333f;
constexpr float kTaylorB = 0.4f;
constexpr float kTaylorC = 0.42857142857142857143f;
constexpr float kTaylorD = 0.44444444444444444444f;
constexpr float kTaylorDD = 0.45454545454545454545f;
constexpr float kTaylorE = 1.33333333333333333333f;
constexpr float kTaylorF = 2.4f;
constexpr float kTaylorG = 3.42857142857142857143f;
constexpr float kTaylorH = 4.44444444444444444444f;
constexpr float kTaylorHH = 5.45454545454545454545f;

constexpr unsigned kFullMask = 0xffffffffu;

// ------------------------------------------------------------------------------------------------
// Clash damping: softened Coulomb and Lennard-Jones cores (Potential/soft_core_potentials.tpp:
// 30-52 and 140-180, as the clash-forgiving GPU kernels apply them,
// nonbonded_potential_tilegroups.cui:536-602)
// ------------------------------------------------------------------------------------------------
// Clash distance and sigma ratio of a molecule in minimization cycle `cycle` of a damping over
// `cycles` cycles (both shrink linearly to zero, hpc_minimization.cu:268-272); cycle < 0: the
// base values unscaled
__device__ __forceinline__ float2 clashScaled(float distance, float ratio, int cycles, int cycle) {
  if (cycle < 0) {
    return make_float2(distance, ratio);
  }
  if (cycle >= cycles) {
    return make_float2(0.0f, 0.0f);
  }
  const double progress = static_cast<double>(cycles - cycle) / static_cast<double>(cycles);
  return make_float2(static_cast<float>(static_cast<double>(distance) * progress),
                     static_cast<float>(static_cast<double>(ratio) * progress));
}

// Constants of the quadratic Coulomb core for a clash distance cd > 0: below cd the pair energy
// is qiqj (a (r + 1)^2 + b), continuous in value and slope with qiqj / r at cd
__device__ __forceinline__ float2 quadraticCore(float cd) {
  if (cd <= 0.0f) {
    return make_float2(0.0f, 0.0f);
  }
  const float a = -0.5f / (cd * cd * (cd + 1.0f));
  return make_float2(a, 1.0f / cd - a * (cd + 1.0f) * (cd + 1.0f));
}

// Coulomb and Lennard-Jones terms of one pair with softened cores: the quadratic Coulomb core
// (constants qc from quadraticCore) below the clash distance cd, the quartic Lennard-Jones core
// below ratio x sigma, sigma = (A / B)^(1/6) (none where B <= 1e-6).  Adds the energies to
// *e_elec and *e_vdw and returns the force factor (force on j = factor x (r_j - r_i)).
__device__ __forceinline__ float softCorePair(float r, float invr, float qiqj, float lja,
                                              float ljb, float cd, float2 qc, float ratio,
                                              float* e_elec, float* e_vdw) {
  float fmag;
  if (r < cd) {
    const float rp = r + 1.0f;
    *e_elec = __fadd_rn(*e_elec, __fmul_rn(qiqj, fmaf(qc.x * rp, rp, qc.y)));
    fmag = (r > 1.0e-10f) ? qiqj * (2.0f * qc.x + 2.0f * qc.x * invr) : 0.0f;
  }
  else {
    *e_elec = __fadd_rn(*e_elec, __fmul_rn(qiqj, invr));
    fmag = -(qiqj * invr * invr * invr);
  }
  const float rl = (ljb > 1.0e-6f) ? ratio * sqrtf(cbrtf(__fdividef(lja, ljb))) : 0.0f;
  if (r < rl) {
    const float il = 1.0f / rl;
    const float il2 = il * il;
    const float il6 = il2 * il2 * il2;
    const float a = ((6.0f * ljb - 12.0f * lja * il6) * il * il6) /
                    (((4.0f * rl + 12.0f) * rl + 12.0f) * rl + 4.0f);
    const float rlp = rl + 1.0f;
    const float rlp2 = rlp * rlp;
    const float b = (lja * il6 - ljb) * il6 - a * rlp2 * rlp2;
    const float rp = r + 1.0f;
    const float a3 = a * rp * rp * rp;
    *e_vdw = __fadd_rn(*e_vdw, fmaf(a3, rp, b));
    if (r > 1.0e-10f) {
      fmag += 4.0f * a3 * invr;
    }
  }
  else {
    const float invr2 = invr * invr;
    const float invr4 = invr2 * invr2;
    *e_vdw = __fadd_rn(*e_vdw, __fmul_rn(__fsub_rn(__fmul_rn(__fmul_rn(lja, invr4), invr4),
                                                   __fmul_rn(ljb, invr2)), invr4));
    fmag += (6.0f * ljb - 12.0f * lja * invr4 * invr2) * invr4 * invr4;
  }
  return fmag;
}

// Valence geometry in FP64 (the angle, dihedral and 1-4 terms of both precision modes)
__device__ __forceinline__ double3 sub3d(double3 a, double3 b) {
  return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double dot3d(double3 a, double3 b) {
  return fma(a.x, b.x, fma(a.y, b.y, a.z * b.z));
}
__device__ __forceinline__ double3 cross3d(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// valence_potential.tpp: below this squared cosine between consecutive dihedral bonds the force
// divides by the sine squared; above it (near-collinear atoms) it takes the fixed reciprocal
constexpr double kAsymptoticToOne = 0.99999904632568359375;
constexpr double kInvOneMinusAsymptote = 1048576.0;

// Softened cores in FP64 (Potential/soft_core_potentials.tpp:30-52, 140-180; softCorePair in
// double)
// Quadratic Coulomb core below cd: qiqj (a (r + 1)^2 + b), continuous in value and slope
__device__ __forceinline__ double2 quadraticCore64(double cd) {
  if (cd <= 0.0) {
    return make_double2(0.0, 0.0);
  }
  const double a = -0.5 / (cd * cd * (cd + 1.0));
  return make_double2(a, 1.0 / cd - a * (cd + 1.0) * (cd + 1.0));
}

// Coulomb and Lennard-Jones energies of one pair with softened cores added to *e_elec, *e_vdw;
// returns the force factor (force on j = factor x (r_j - r_i))
__device__ __forceinline__ double softCorePair64(double r, double invr, double qiqj, double lja,
                                                 double ljb, double cd, double2 qc, double ratio,
                                                 double* e_elec, double* e_vdw) {
  double fmag;
  if (r < cd) {
    const double rp = r + 1.0;
    *e_elec += qiqj * (qc.x * rp * rp + qc.y);
    fmag = (r > 1.0e-10) ? qiqj * (2.0 * qc.x + 2.0 * qc.x * invr) : 0.0;
  }
  else {
    *e_elec += qiqj * invr;
    fmag = -(qiqj * invr * invr * invr);
  }
  const double rl = (ljb > 1.0e-6) ? ratio * pow(lja / ljb, 1.0 / 6.0) : 0.0;
  if (r < rl) {
    const double il = 1.0 / rl;
    const double il2 = il * il;
    const double il6 = il2 * il2 * il2;
    const double a = ((6.0 * ljb - 12.0 * lja * il6) * il * il6) /
                     (((4.0 * rl + 12.0) * rl + 12.0) * rl + 4.0);
    const double rlp = rl + 1.0;
    const double rlp2 = rlp * rlp;
    const double b = (lja * il6 - ljb) * il6 - a * rlp2 * rlp2;
    const double rp = r + 1.0;
    const double a3 = a * rp * rp * rp;
    *e_vdw += a3 * rp + b;
    if (r > 1.0e-10) {
      fmag += 4.0 * a3 * invr;
    }
  }
  else {
    const double invr2 = invr * invr;
    const double invr4 = invr2 * invr2;
    *e_vdw += (lja * invr4 * invr4 - ljb * invr2) * invr4;
    fmag += (6.0 * ljb - 12.0 * lja * invr4 * invr2) * invr4 * invr4;
  }
  return fmag;
}


// Packed FP32 pairs (Blackwell FFMA2 / FADD2 / FMUL2): two pairs of one lane in one instruction
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }


// HCT descreening of an atom of offset radius rho by a neighbour of screened radius sj at
// distance r (invr = 1/r), for two (r, rho, sj) combinations at once in packed FP32; returns the
// amounts psi decreases by.
//
// Beyond r = 4 sj the reference's Taylor series applies (nonbonded_potential.tpp:590-596).
// Closer in, the three closed forms the reference selects by overlap case (no overlap, partial
// overlap, atom inside the neighbour's sphere: nonbonded_potential.tpp:597-628) are one
// expression in U = r + sj and L = max(rho, |r - sj|):
//   I = 1/2 [1/L - 1/U + (sj^2 - r^2)/(4r) (1/L^2 - 1/U^2) + ln(L/U) / (2r)]
//       + (1/rho - 1/L) when rho < sj - r,
// and I = 0 when rho >= U.  One formula instead of four keeps a warp on at most two paths; the
// inside case is rare, so a branch there beats a reciprocal per pair.  The closed form cancels
// to a small remainder near r = 4 sj, so ln(L / U) needs an accurate absolute value: the fast
// hardware logarithm (__logf) errs by about 1e-7 absolute with a consistent sign, which biased
// every atom's psi by -6.5e-7 relative and the GB energy by +1.1e-6 relative (1,024 molecules
// of 16-256 atoms); logf removes the bias (psi -7.6e-8, GB energy 1.0e-7).
__device__ __forceinline__ float2 hctIntegral2(float2 r, float2 r2, float2 invr, float2 rho,
                                               float2 sj) {
  const bool far_x = r.x > 4.0f * sj.x;
  const bool far_y = r.y > 4.0f * sj.y;
  float2 vf = f2(0.0f);
  float2 vn = f2(0.0f);
  if (far_x || far_y) {
    const float2 invr2 = mul2(invr, invr);
    const float2 t = mul2(mul2(sj, sj), invr2);
    float2 dumbo = fma2(t, f2(kTaylorDD), f2(kTaylorD));
    dumbo = fma2(t, dumbo, f2(kTaylorC));
    dumbo = fma2(t, dumbo, f2(kTaylorB));
    dumbo = fma2(t, dumbo, f2(kTaylorA));
    vf = mul2(mul2(mul2(sj, t), invr2), dumbo);
  }
  if (!(far_x && far_y)) {
    const float2 u = add2(r, sj);
    const float2 rms = sub2(r, sj);
    const float2 l = f2(fmaxf(rho.x, fabsf(rms.x)), fmaxf(rho.y, fabsf(rms.y)));
    const float2 lu = mul2(l, u);
    const float2 inv_lu = f2(__fdividef(1.0f, lu.x), __fdividef(1.0f, lu.y));
    const float2 il = mul2(u, inv_lu);
    const float2 iu = mul2(l, inv_lu);
    const float2 dlu = sub2(il, iu);
    const float2 liu = mul2(l, iu);
    const float2 lg = f2(logf(liu.x), logf(liu.y));
    const float2 q = mul2(mul2(mul2(f2(0.25f), sub2(mul2(sj, sj), r2)), invr), dlu);
    float2 v = add2(fma2(q, add2(il, iu), dlu), mul2(mul2(f2(0.5f), invr), lg));
    if (rho.x < -rms.x) {
      v.x += 2.0f * (__fdividef(1.0f, rho.x) - il.x);
    }
    if (rho.y < -rms.y) {
      v.y += 2.0f * (__fdividef(1.0f, rho.y) - il.y);
    }
    vn = f2((rho.x < u.x) ? 0.5f * v.x : 0.0f, (rho.y < u.y) ? 0.5f * v.y : 0.0f);
  }
  return f2(far_x ? vf.x : vn.x, far_y ? vf.y : vn.y);
}

// Radial derivative of the HCT integral, -(1/r) dI/dr, the factor the reference multiplies by
// the chain-rule dE/dR (nonbonded_potential.tpp:1116-1165), from the same unified expression
// (lambda = dL/dr: 1 without overlap, 0 on partial overlap, -1 inside the neighbour):
//   dI/dr = 1/2 [-lambda/L^2 + 1/U^2 + q'(1/L^2 - 1/U^2) + 2q (1/U^3 - lambda/L^3)
//                + (lambda/L - 1/U - ln(L/U)/r) / (2r)] - 1/L^2 (inside),
// q = (sj^2 - r^2)/(4r), q' = dq/dr.
__device__ __forceinline__ float hctDerivative(float r, float r2, float invr, float rho,
                                               float sj) {
  const float invr2 = invr * invr;
  if (r > 4.0f * sj) {
    const float t = sj * sj * invr2;
    const float dumbo = kTaylorE + t * (kTaylorF + t * (kTaylorG + t * (kTaylorH + t * kTaylorHH)));
    return t * sj * invr2 * invr2 * dumbo;
  }
  const float u = r + sj;
  const float rms = r - sj;
  const float l = fmaxf(rho, fabsf(rms));
  const float lam = (rms >= rho) ? 1.0f : ((-rms > rho) ? -1.0f : 0.0f);
  const float inv_lu = __fdividef(1.0f, l * u);
  const float il = u * inv_lu;
  const float iu = l * inv_lu;
  const float il2 = il * il;
  const float iu2 = iu * iu;
  const float q = 0.25f * (sj * sj - r2) * invr;
  const float dq = -0.25f * fmaf(sj * sj, invr2, 1.0f);
  float di = -lam * il2 + iu2 + dq * (il2 - iu2) + 2.0f * q * (iu2 * iu - lam * il2 * il) +
             0.5f * invr * (lam * il - iu - invr * logf(l * iu));
  di = 0.5f * di - ((-rms > rho) ? il2 : 0.0f);
  return (rho < u) ? -di * invr : 0.0f;
}

// The HCT integral and its radial derivative together, for both directions of one pair (x for
// (rho.x, sj.x), y for (rho.y, sj.y)): the Taylor forms share t = (sj / r)^2, the closed forms
// share the reciprocals and the logarithm.
__device__ __forceinline__ void hctBoth2(float r, float r2, float invr, float2 rho, float2 sj,
                                         float2* integral, float2* deriv) {
  const float invr2 = invr * invr;
  const bool far_x = r > 4.0f * sj.x;
  const bool far_y = r > 4.0f * sj.y;
  const float2 sj2 = mul2(sj, sj);
  float2 vfi = f2(0.0f), vfd = f2(0.0f), vni = f2(0.0f), vnd = f2(0.0f);
  if (far_x || far_y) {
    const float2 t = mul2(sj2, f2(invr2));
    float2 di = fma2(t, f2(kTaylorDD), f2(kTaylorD));
    di = fma2(t, di, f2(kTaylorC));
    di = fma2(t, di, f2(kTaylorB));
    di = fma2(t, di, f2(kTaylorA));
    float2 dd = fma2(t, f2(kTaylorHH), f2(kTaylorH));
    dd = fma2(t, dd, f2(kTaylorG));
    dd = fma2(t, dd, f2(kTaylorF));
    dd = fma2(t, dd, f2(kTaylorE));
    const float2 tsr = mul2(mul2(sj, t), f2(invr2));
    vfi = mul2(tsr, di);
    vfd = mul2(mul2(tsr, f2(invr2)), dd);
  }
  if (!(far_x && far_y)) {
    const float2 u = add2(f2(r), sj);
    const float2 rms = sub2(f2(r), sj);
    const float2 l = f2(fmaxf(rho.x, fabsf(rms.x)), fmaxf(rho.y, fabsf(rms.y)));
    const bool in_x = -rms.x > rho.x;      // inside the neighbour's sphere
    const bool in_y = -rms.y > rho.y;
    const float2 lu = mul2(l, u);
    const float2 inv_lu = f2(__fdividef(1.0f, lu.x), __fdividef(1.0f, lu.y));
    const float2 il = mul2(u, inv_lu);
    const float2 iu = mul2(l, inv_lu);
    const float2 liu = mul2(l, iu);
    const float2 lg = f2(logf(liu.x), logf(liu.y));
    const float2 s2mr2 = sub2(sj2, f2(r2));
    // the integral
    const float2 dlu = sub2(il, iu);
    const float2 q = mul2(mul2(f2(0.25f * invr), s2mr2), dlu);
    float2 v = add2(fma2(q, add2(il, iu), dlu), mul2(f2(0.5f * invr), lg));
    if (in_x) {
      v.x += 2.0f * (__fdividef(1.0f, rho.x) - il.x);
    }
    if (in_y) {
      v.y += 2.0f * (__fdividef(1.0f, rho.y) - il.y);
    }
    vni = f2((rho.x < u.x) ? 0.5f * v.x : 0.0f, (rho.y < u.y) ? 0.5f * v.y : 0.0f);
    // its derivative, lambda = dL/dr
    const float2 lam = f2((rms.x >= rho.x) ? 1.0f : (in_x ? -1.0f : 0.0f),
                          (rms.y >= rho.y) ? 1.0f : (in_y ? -1.0f : 0.0f));
    const float2 il2 = mul2(il, il);
    const float2 iu2 = mul2(iu, iu);
    const float2 q2 = mul2(f2(0.5f * invr), s2mr2);
    const float2 dq = mul2(f2(-0.25f), fma2(sj2, f2(invr2), f2(1.0f)));
    const float2 lil2 = mul2(lam, il2);
    float2 dv = sub2(iu2, lil2);
    dv = fma2(dq, sub2(il2, iu2), dv);
    dv = fma2(q2, sub2(mul2(iu2, iu), mul2(lil2, il)), dv);
    dv = fma2(f2(0.5f * invr), sub2(sub2(mul2(lam, il), iu), mul2(f2(invr), lg)), dv);
    dv = sub2(mul2(f2(0.5f), dv), f2(in_x ? il2.x : 0.0f, in_y ? il2.y : 0.0f));
    const float2 w = mul2(dv, f2(-invr));
    vnd = f2((rho.x < u.x) ? w.x : 0.0f, (rho.y < u.y) ? w.y : 0.0f);
  }
  *integral = f2(far_x ? vfi.x : vni.x, far_y ? vfi.y : vni.y);
  *deriv = f2(far_x ? vfd.x : vnd.x, far_y ? vfd.y : vnd.y);
}

// Neck GB (Mongan's neck between two spheres, nonbonded_potential.tpp:678-702, 1219-1245): pairs
// closer than rho_i + rho_j + 2 offset + cutoff add scale * V / (1 + m^2 + 0.3 m^6), m = r - S,
// to the descreening, with V and S looked up for the pair's neck indices
struct NeckGb {
  const float* sep;
  const float* val;
  int size;
  float scale;
  float reach;     // 2 offset + cutoff: the pair takes the neck term when r < rho_i + rho_j + reach
  __device__ explicit NeckGb(const DevSynthesis &d) :
      sep(d.neck_sep), val(d.neck_val), size(d.neck_size), scale(d.neck_scale),
      reach(2.0f * d.gb_offset + d.neck_cut) {}
  // the amount psi of the atom with index ni decreases by from the atom with index nj
  __device__ __forceinline__ float integral(int ni, int nj, float r) const {
    const int t = size * nj + ni;
    const float m = r - __ldg(&sep[t]);
    const float m2 = m * m;
    return __fdividef(scale * __ldg(&val[t]), 1.0f + m2 + 0.3f * m2 * m2 * m2);
  }
  // the same and its radial derivative factor -(1/r) dI/dr, as hctDerivative
  __device__ __forceinline__ float both(int ni, int nj, float r, float invr, float* deriv) const {
    const int t = size * nj + ni;
    const float m = r - __ldg(&sep[t]);
    const float m2 = m * m;
    const float v = scale * __ldg(&val[t]);
    const float inv_den = __fdividef(1.0f, 1.0f + m2 + 0.3f * m2 * m2 * m2);
    *deriv = (2.0f * m + 1.8f * m2 * m2 * m) * v * inv_den * inv_den * invr;
    return v * inv_den;
  }
};

// Shared-memory layout of one work unit
struct UnitSmem {
  float4* pa;       // x_hi, y_hi, z_hi, pass payload w1
  float4* pb;       // x_lo, y_lo, z_lo, pass payload w2
  float4* prm;      // charge * sqrt(k_Coulomb), Lennard-Jones code (int bits), rho, s * rho
  float2* gbv;      // 1 / effective radius; y: Lennard-Jones code bits in pass 2, dE/dR after
                    // the chain rule
  int* fx;          // int63 force accumulators: primary
  int* fy;
  int* fz;
  int* fxo;         // overflow
  int* fyo;
  int* fzo;
  int* psi;         // int63 psi accumulator, 2^kPsiBits
  int* psio;
  int* de;          // int63 dE/dR accumulator, 2^kDeijdaBits
  int* deo;
  int* neck;        // neck GB table index of the atom
  float2* lj;       // Lennard-Jones tables of the unit's molecules (standard, then 1-4)
  unsigned long long* nrg;   // per unit molecule energies
  int* sys;         // molecule index
  int* slot0;       // first slot of the molecule
  int* natom;
  int* ljbase;      // prefix sums of the molecules' table sizes (kMaxUnitSystems + 1)
  int* tile0;       // prefix sums (kMaxUnitSystems + 1 entries each)
  int* bchunk0;     // valence work in chunks of 32 terms that never straddle two molecules
  int* achunk0;
  int* dchunk0;
  float2* clash;    // per unit molecule: clash distance and sigma ratio of this evaluation
};

__host__ __device__ inline size_t alignUp(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Raise a kernel's dynamic shared-memory limit to the device's opt-in maximum, once per kernel and
// device (the attribute belongs to the function on the current device); launches then pass only
// their own size, and the per-system drop-in, a launch per molecule, pays no attribute call
template <class K>
cudaError_t allowLargeSmem(K kern) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kern), dev);
  if (done.count(key) != 0) return cudaSuccess;
  int optin = 0;
  err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (err != cudaSuccess) return err;
  // static and dynamic shared memory together may not exceed the opt-in maximum
  cudaFuncAttributes attr;
  err = cudaFuncGetAttributes(&attr, kern);
  if (err != cudaSuccess) return err;
  err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - static_cast<int>(attr.sharedSizeBytes));
  if (err == cudaSuccess) {
    done.insert(key);
  }
  else {
    cudaGetLastError();   // reported here, not left for the next launch check to find
  }
  return err;
}

constexpr int kSlotBytes = 3 * 16 + 8 + 11 * 4;

// Dynamic shared memory of one work unit's evaluation: max_slots atom slots, max_lj table entries
__host__ __device__ inline size_t unitSmemBytes(int max_slots, int max_lj,
                                                int max_sys = kMaxUnitSystems) {
  size_t b = static_cast<size_t>(kSlotBytes) * max_slots;
  b = alignUp(b, 16);
  b += sizeof(float2) * max_lj;
  b = alignUp(b, 16);
  b += sizeof(unsigned long long) * max_sys * kNrgStride;
  b += sizeof(float2) * max_sys;
  b += sizeof(int) * (3 * max_sys + 5 * (max_sys + 1));
  return alignUp(b, 16);
}

__device__ UnitSmem carveSmem(char* base, int max_slots, int max_lj,
                              int max_sys = kMaxUnitSystems) {
  UnitSmem s;
  size_t off = 0;
  s.pa = reinterpret_cast<float4*>(base + off); off += sizeof(float4) * max_slots;
  s.pb = reinterpret_cast<float4*>(base + off); off += sizeof(float4) * max_slots;
  s.prm = reinterpret_cast<float4*>(base + off); off += sizeof(float4) * max_slots;
  s.gbv = reinterpret_cast<float2*>(base + off); off += sizeof(float2) * max_slots;
  int* ip = reinterpret_cast<int*>(base + off);
  s.fx = ip; ip += max_slots;
  s.fy = ip; ip += max_slots;
  s.fz = ip; ip += max_slots;
  s.fxo = ip; ip += max_slots;
  s.fyo = ip; ip += max_slots;
  s.fzo = ip; ip += max_slots;
  s.psi = ip; ip += max_slots;
  s.psio = ip; ip += max_slots;
  s.de = ip; ip += max_slots;
  s.deo = ip; ip += max_slots;
  s.neck = ip; ip += max_slots;
  off = alignUp(off + 11 * sizeof(int) * max_slots, 16);
  s.lj = reinterpret_cast<float2*>(base + off); off += sizeof(float2) * max_lj;
  off = alignUp(off, 16);
  s.nrg = reinterpret_cast<unsigned long long*>(base + off);
  off += sizeof(unsigned long long) * max_sys * kNrgStride;
  s.clash = reinterpret_cast<float2*>(base + off);
  off += sizeof(float2) * max_sys;
  int* q = reinterpret_cast<int*>(base + off);
  s.sys = q; q += max_sys;
  s.slot0 = q; q += max_sys;
  s.natom = q; q += max_sys;
  s.ljbase = q; q += max_sys + 1;
  s.tile0 = q; q += max_sys + 1;
  s.bchunk0 = q; q += max_sys + 1;
  s.achunk0 = q; q += max_sys + 1;
  s.dchunk0 = q; q += max_sys + 1;
  return s;
}

// The threads that evaluate one work unit together: a whole block, or a single warp (small
// molecules, where block-wide barriers would cost more than the work between them)
struct BlockTeam {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ int warp() const { return threadIdx.x >> 5; }
  __device__ __forceinline__ int warps() const { return blockDim.x >> 5; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ bool any(bool p) const { return __syncthreads_or(p) != 0; }
};

struct WarpTeam {
  __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ int warp() const { return 0; }
  __device__ __forceinline__ int warps() const { return 1; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  __device__ __forceinline__ bool any(bool p) const { return __any_sync(0xffffffffu, p) != 0; }
};

// Index of the unit molecule that owns position pos of a prefix-sum array of n + 1 entries
__device__ __forceinline__ int findOwner(const int* prefix, int n, int pos) {
  int k = 0;
  while (k + 1 < n && prefix[k + 1] <= pos) {
    k++;
  }
  return k;
}

// Tile (I, J), I >= J, of the lower triangle from its index within the molecule
__device__ __forceinline__ void tileCoordinates(int local, int* ti, int* tj) {
  int i = static_cast<int>((sqrtf(8.0f * local + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > local) i--;
  while ((i + 1) * (i + 2) / 2 <= local) i++;
  *ti = i;
  *tj = local - i * (i + 1) / 2;
}

__device__ __forceinline__ float3 pairDelta(const float4 a_i, const float4 b_i, const float4 a_j,
                                            const float4 b_j) {
  return make_float3((a_j.x - a_i.x) + (b_j.x - b_i.x), (a_j.y - a_i.y) + (b_j.y - b_i.y),
                     (a_j.z - a_i.z) + (b_j.z - b_i.z));
}

__device__ __forceinline__ void addForce(const UnitSmem &s, int slot, float fx, float fy, float fz,
                                         float scale) {
  atomicAddInt63(fx * scale, &s.fx[slot], &s.fxo[slot]);
  atomicAddInt63(fy * scale, &s.fy[slot], &s.fyo[slot]);
  atomicAddInt63(fz * scale, &s.fz[slot], &s.fzo[slot]);
}

// Warp-wide int64 sum, result in every lane
__device__ __forceinline__ long long warpSum(long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(kFullMask, v, o);
  }
  return v;
}

// A tile's energy in the output fixed-point format: the lanes' FP64 sums added by an xor
// butterfly (every lane adds the same two values at every level, so all lanes hold the same bits
// and the total does not depend on which warp ran the tile), then rounded once.  Rounding each
// lane's share instead loses the pairs of distant tiles, whose per-lane sums fall below one unit
// of 2^-26 kcal/mol (1.6e-6 of the Lennard-Jones energy of a 2,100-atom chain), and an integer
// accumulator finer than the output overflows on clashing starting structures (1.6e7 kcal/mol).
__device__ __forceinline__ long long tileEnergy(double v, float nrg_scale) {
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(kFullMask, v, o);
  }
  return __double2ll_rn(v * static_cast<double>(nrg_scale));
}

// Warp-reduce one scaled energy per lane (all lanes in one molecule) into its slot
__device__ __forceinline__ void warpEnergy(const UnitSmem &s, int k, int slot, float e,
                                           float scale) {
  const long long v = warpSum(__float2ll_rn(e * scale));
  if ((threadIdx.x & 31) == 0 && v != 0) {
    atomicAdd(&s.nrg[k * kNrgStride + slot], static_cast<unsigned long long>(v));
  }
}

// Coordinate difference b - a from the hi / lo representation of two slots
__device__ __forceinline__ float3 slotDelta(const UnitSmem &s, int a, int b) {
  return pairDelta(s.pa[a], s.pb[a], s.pa[b], s.pb[b]);
}

// ------------------------------------------------------------------------------------------------
// Valence terms (Potential/valence_potential.tpp).  Warps take chunks of 32 terms of one molecule,
// so each chunk's energies reduce across the warp into a single shared-memory update.
// ------------------------------------------------------------------------------------------------
// Where valence terms read their atoms and put forces and energies: a work unit's shared memory
struct SmemValence {
  const UnitSmem &s;
  const int* bchunk0;
  const int* achunk0;
  const int* dchunk0;
  const int* sys;
  const int* slot0;
  int begin;
  int stride;
  __device__ SmemValence(const UnitSmem &s_in, int begin_in, int stride_in) :
      s(s_in), bchunk0(s_in.bchunk0), achunk0(s_in.achunk0), dchunk0(s_in.dchunk0),
      sys(s_in.sys), slot0(s_in.slot0), begin(begin_in), stride(stride_in) {}
  __device__ __forceinline__ int chunkBegin() const { return begin; }
  __device__ __forceinline__ int chunkStride() const { return stride; }
  __device__ __forceinline__ float4 pa(int i) const { return s.pa[i]; }
  __device__ __forceinline__ float4 pb(int i) const { return s.pb[i]; }
  __device__ __forceinline__ float4 prm(int i) const { return s.prm[i]; }
  __device__ __forceinline__ float3 delta(int a, int b) const { return slotDelta(s, a, b); }
  __device__ __forceinline__ void force(int i, float fx, float fy, float fz, float scale) const {
    addForce(s, i, fx, fy, fz, scale);
  }
  __device__ __forceinline__ void energy(int k, int slot, float e, float scale) const {
    warpEnergy(s, k, slot, e, scale);
  }
  // exact coordinates of a slot: the hi + lo float pair summed in double
  __device__ __forceinline__ double3 pos64(int i) const {
    const float4 a = s.pa[i];
    const float4 b = s.pb[i];
    return make_double3(static_cast<double>(a.x) + static_cast<double>(b.x),
                        static_cast<double>(a.y) + static_cast<double>(b.y),
                        static_cast<double>(a.z) + static_cast<double>(b.z));
  }
  __device__ __forceinline__ void force64(int i, double fx, double fy, double fz,
                                          float scale) const {
    addForce(s, i, static_cast<float>(fx), static_cast<float>(fy), static_cast<float>(fz),
             scale);
  }
  __device__ __forceinline__ void energy64(int k, int slot, double e, float scale) const {
    const long long v = warpSum(__double2ll_rn(e * static_cast<double>(scale)));
    if ((threadIdx.x & 31) == 0 && v != 0) {
      atomicAdd(&s.nrg[k * kNrgStride + slot], static_cast<unsigned long long>(v));
    }
  }
  __device__ __forceinline__ float2 clash(int k) const { return s.clash[k]; }
  // the molecule's 1-4 table follows its standard table in shared memory
  __device__ __forceinline__ float2 lj14(int code_i, int code_l, int nt) const {
    return s.lj[(code_i & 0xffff) + (code_l >> 16) + nt * nt];
  }
};

template <bool FORCE, bool ENERGY, class V, bool CLASH = false>
__device__ void valenceTerms(const DevSynthesis &d, const V &v, int nsys_u) {
  const float fs = d.frc_scale;
  const float es = d.nrg_scale;
  const int lane = threadIdx.x & 31;

  // bonds, valence_potential.tpp:9-97; the equilibrium length is a float pair so that r - r0
  // loses nothing to the rounding of r0, and the bond length itself is an unevaluated pair
  for (int c = v.chunkBegin(); c < v.bchunk0[nsys_u]; c += v.chunkStride()) {
    const int k = findOwner(v.bchunk0, nsys_u, c);
    const int sysid = v.sys[k];
    const int t = (c - v.bchunk0[k]) * 32 + lane;
    const int nterm = d.bond_start[sysid + 1] - d.bond_start[sysid];
    float e = 0.0f;
    if (t < nterm) {
      const uint4 rec = d.bonds[d.bond_start[sysid] + t];
      const int ia = v.slot0[k] + static_cast<int>(rec.x & 0xffffu);
      const int ja = v.slot0[k] + static_cast<int>(rec.x >> 16);
      const float keq = __uint_as_float(rec.y);
      const float leq_hi = __uint_as_float(rec.z);
      const float leq_lo = __uint_as_float(rec.w);
      const float4 ai = v.pa(ia), aj = v.pa(ja), bi = v.pb(ia), bj = v.pb(ja);
      const float av[3] = {aj.x, aj.y, aj.z};
      const float bv[3] = {ai.x, ai.y, ai.z};
      const float lav[3] = {bj.x, bj.y, bj.z};
      const float lbv[3] = {bi.x, bi.y, bi.z};
      float dh[3], dlo[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float sdiff = av[q] - bv[q];
        const float bb = sdiff - av[q];
        const float err = (av[q] - (sdiff - bb)) + (-bv[q] - bb);
        const float lo = err + (lav[q] - lbv[q]);
        dh[q] = sdiff + lo;
        dlo[q] = lo - (dh[q] - sdiff);
      }
      float r2h = dh[0] * dh[0];
      float r2l = fmaf(dh[0], dh[0], -r2h) + 2.0f * dh[0] * dlo[0];
#pragma unroll
      for (int q = 1; q < 3; q++) {
        const float p = dh[q] * dh[q];
        const float pe = fmaf(dh[q], dh[q], -p) + 2.0f * dh[q] * dlo[q];
        const float sum = r2h + p;
        const float bvv = sum - r2h;
        r2l += ((r2h - (sum - bvv)) + (p - bvv)) + pe;
        r2h = sum;
      }
      const float r = sqrtf(r2h);
      const float r_lo = (fmaf(-r, r, r2h) + r2l) / (2.0f * r);
      const float dl = ((r - leq_hi) + r_lo) - leq_lo;
      if (FORCE) {
        const float fmag = 2.0f * keq * dl / r;
        v.force(ia, fmag * dh[0], fmag * dh[1], fmag * dh[2], fs);
        v.force(ja, -fmag * dh[0], -fmag * dh[1], -fmag * dh[2], fs);
      }
      e = __fmul_rn(__fmul_rn(keq, dl), dl);
    }
    if (ENERGY) {
      v.energy(k, kBond, e, es);
    }
  }

  // angles, valence_potential.tpp:170-288, in FP64 from the exact coordinates: a near-linear
  // angle's force divides by sin(theta), which FP32 deltas and cross products only give to
  // about 1e-7 absolute.  theta - theta0 comes from rotating (cos, sin) of theta, taken from the
  // dot and cross products, by theta0: well conditioned everywhere.
  for (int c = v.chunkBegin(); c < v.achunk0[nsys_u]; c += v.chunkStride()) {
    const int k = findOwner(v.achunk0, nsys_u, c);
    const int sysid = v.sys[k];
    const int t = (c - v.achunk0[k]) * 32 + lane;
    const int nterm = d.angl_start[sysid + 1] - d.angl_start[sysid];
    double e = 0.0;
    if (t < nterm) {
      const uint4 rec = d.angles[d.angl_start[sysid] + t];
      const double4 prm = d.angl64[d.angl_start[sysid] + t];   // k, cos, sin, theta0
      const int ia = v.slot0[k] + static_cast<int>(rec.x & 0xffffu);
      const int ja = v.slot0[k] + static_cast<int>(rec.x >> 16);
      const int ka = v.slot0[k] + static_cast<int>(rec.y);
      const double3 pj = v.pos64(ja);
      const double3 ba = sub3d(v.pos64(ia), pj);
      const double3 bc = sub3d(v.pos64(ka), pj);
      // reciprocal square roots instead of divisions and square roots (FP64 divisions are long
      // instruction sequences): 1 / sin(theta) = |ba| |bc| / |ba x bc|
      const double mgba = dot3d(ba, ba);
      const double mgbc = dot3d(bc, bc);
      const double inv_ba = rsqrt(mgba);
      const double inv_bc = rsqrt(mgbc);
      const double invbabc = inv_ba * inv_bc;
      const double3 cr = cross3d(ba, bc);
      const double cr2 = dot3d(cr, cr);
      const double inv_cr = rsqrt(cr2);
      const double sth = cr2 * inv_cr * invbabc;
      const double cth = dot3d(ba, bc) * invbabc;
      const double dtheta = atan2(fma(sth, prm.y, -cth * prm.z), fma(cth, prm.y, sth * prm.z));
      if (FORCE) {
        const double dA = -2.0 * prm.x * dtheta * inv_cr * ((mgba * inv_ba) * (mgbc * inv_bc));
        const double sqba = dA * inv_ba * inv_ba;
        const double sqbc = dA * inv_bc * inv_bc;
        const double mbabc = dA * invbabc;
        const double adx = bc.x * mbabc - cth * ba.x * sqba;
        const double ady = bc.y * mbabc - cth * ba.y * sqba;
        const double adz = bc.z * mbabc - cth * ba.z * sqba;
        const double cdx = ba.x * mbabc - cth * bc.x * sqbc;
        const double cdy = ba.y * mbabc - cth * bc.y * sqbc;
        const double cdz = ba.z * mbabc - cth * bc.z * sqbc;
        v.force64(ia, -adx, -ady, -adz, fs);
        v.force64(ja, adx + cdx, ady + cdy, adz + cdz, fs);
        v.force64(ka, -cdx, -cdy, -cdz, fs);
      }
      e = prm.x * dtheta * dtheta;
    }
    if (ENERGY) {
      v.energy64(k, kAngle, e, es);
    }
  }

  // dihedrals with attached 1-4 pairs, valence_potential.tpp:359-578, 1288-1420, in FP64 from
  // the exact coordinates.  The signed angle is carried as (cos, sin) from x = (ab x bc) .
  // (bc x cd) and y = |bc| ab . (bc x cd), the angle STORMM's acos / arcsine route gives
  // (Math/rounding.tpp:25-80) without its ill conditioning near 0 and pi; cos(n theta - phase)
  // and sin(n theta - phase) follow from the multiple-angle recurrence for integer
  // periodicities.  1 + cos(psi) cancels near psi = pi (impropers, and propers near their
  // minimum); there sin^2(psi) / (1 - cos(psi)) gives the same value without the cancellation.
  for (int c = v.chunkBegin(); c < v.dchunk0[nsys_u]; c += v.chunkStride()) {
    const int k = findOwner(v.dchunk0, nsys_u, c);
    const int sysid = v.sys[k];
    const int t = (c - v.dchunk0[k]) * 32 + lane;
    const int nterm = d.dihe_start[sysid + 1] - d.dihe_start[sysid];
    double e_prop = 0.0, e_impr = 0.0, e_el14 = 0.0, e_lj14 = 0.0;
    if (t < nterm) {
      const int pos = d.dihe_start[sysid] + t;
      const uint4 ra = d.dihe_a[pos];
      const double4 prm = d.dihe64[pos];     // amplitude, cos(phase), sin(phase), periodicity
      const double4 p14 = d.dihe14_64[pos];  // the attached 1-4 pair: q q / scee, A, B, flag
      const int li = static_cast<int>(ra.x & 0xffffu);
      const int ll = static_cast<int>((ra.y >> 16) & 0x7fffu);
      const int ia = v.slot0[k] + li;
      const int ja = v.slot0[k] + static_cast<int>(ra.x >> 16);
      const int ka = v.slot0[k] + static_cast<int>(ra.y & 0xffffu);
      const int la = v.slot0[k] + ll;
      const bool improper = (ra.y & 0x80000000u) != 0u;
      const double3 pi = v.pos64(ia);
      const double3 pj = v.pos64(ja);
      const double3 pk = v.pos64(ka);
      const double3 pl = v.pos64(la);
      const double3 ab = sub3d(pj, pi);
      const double3 bc = sub3d(pk, pj);
      const double3 cd = sub3d(pl, pk);
      // attached 1-4 pair between atoms i and l, its attenuated FP64 parameters stored with
      // the term; evaluated first, so that the atoms' positions are no longer live in the
      // torsion's force, and its force joins the torsion's on atoms i and l (one set of
      // accumulator atomics for both)
      double3 f14 = make_double3(0.0, 0.0, 0.0);
      if (p14.w != 0.0) {
        const double3 dv = sub3d(pl, pi);
        const double qiqj = p14.x;
        const double lja = p14.y;
        const double ljb = p14.z;
        const double invr = rsqrt(dot3d(dv, dv));
        const double invr2 = invr * invr;
        const double invr6 = invr2 * invr2 * invr2;
        const float2 cl = CLASH ? v.clash(k) : make_float2(0.0f, 0.0f);
        double fmag = 0.0;
        if (CLASH && (cl.x > 0.0f || cl.y > 0.0f)) {
          // clash-softened 1-4 pair (valence_potential.tpp:1337-1357)
          fmag = softCorePair64(1.0 / invr, invr, qiqj, lja, ljb, cl.x, quadraticCore64(cl.x),
                                cl.y, &e_el14, &e_lj14);
        }
        else {
          if (FORCE) {
            fmag = -(qiqj * invr * invr2) + (6.0 * ljb - 12.0 * lja * invr6) * invr6 * invr2;
          }
          e_el14 = qiqj * invr;
          e_lj14 = (lja * invr6 - ljb) * invr6;
        }
        f14 = make_double3(fmag * dv.x, fmag * dv.y, fmag * dv.z);
      }
      double3 crabbc = cross3d(ab, bc);
      double3 crbccd = cross3d(bc, cd);
      const double bc2 = dot3d(bc, bc);
      const double invbc = rsqrt(bc2);
      const double mgbc = bc2 * invbc;
      const double xx = dot3d(crabbc, crbccd);
      const double yy = mgbc * dot3d(ab, crbccd);
      const double inv_rr = rsqrt(fma(xx, xx, yy * yy));
      const double c1 = xx * inv_rr;
      const double s1 = yy * inv_rr;
      double cn, sn;
      const double freq = prm.w;
      const int nint = static_cast<int>(freq);
      if (static_cast<double>(nint) == freq && nint >= 1 && nint <= 6) {
        cn = c1;
        sn = s1;
        for (int m = 1; m < nint; m++) {
          const double cnew = cn * c1 - sn * s1;
          sn = sn * c1 + cn * s1;
          cn = cnew;
        }
      }
      else {
        sincos(freq * atan2(yy, xx), &sn, &cn);
      }
      const double cos_sangle = cn * prm.y + sn * prm.z;
      const double sin_sangle = sn * prm.y - cn * prm.z;
      const double opc = (cos_sangle >= 0.0) ? 1.0 + cos_sangle :
                                               sin_sangle * sin_sangle / (1.0 - cos_sangle);
      if (improper) {
        e_impr = prm.x * opc;
      }
      else {
        e_prop = prm.x * opc;
      }
      if (FORCE) {
        const double fr = prm.x * freq * sin_sangle;
        const double ab2 = dot3d(ab, ab);
        const double cd2 = dot3d(cd, cd);
        const double invab = rsqrt(ab2);
        const double invcd = rsqrt(cd2);
        const double mgab = ab2 * invab;
        const double cosb = -dot3d(ab, bc) * invab * invbc;
        const double cosc = -dot3d(bc, cd) * invbc * invcd;
        const double isinb2 = (cosb * cosb < kAsymptoticToOne) ?
                              fr * __drcp_rn(1.0 - cosb * cosb) : fr * kInvOneMinusAsymptote;
        const double isinc2 = (cosc * cosc < kAsymptoticToOne) ?
                              fr * __drcp_rn(1.0 - cosc * cosc) : fr * kInvOneMinusAsymptote;
        const double invabc = invab * invbc;
        const double invbcd = invbc * invcd;
        crabbc = make_double3(crabbc.x * invabc, crabbc.y * invabc, crabbc.z * invabc);
        crbccd = make_double3(crbccd.x * invbcd, crbccd.y * invbcd, crbccd.z * invbcd);
        const double fa = -invab * isinb2;
        const double fb1 = (mgbc - mgab * cosb) * invabc * isinb2;
        const double fb2 = cosc * invbc * isinc2;
        const double fd = -invcd * isinc2;
        // each atom's force goes out as soon as it is formed (fewer doubles live at once); the
        // third atom takes minus the sum of the torsion's other three, (fb2 + fd) cd' -
        // (fa + fb1) ab'
        v.force64(ia, crabbc.x * fa + f14.x, crabbc.y * fa + f14.y, crabbc.z * fa + f14.z, fs);
        v.force64(la, -fd * crbccd.x - f14.x, -fd * crbccd.y - f14.y, -fd * crbccd.z - f14.z, fs);
        v.force64(ja, fb1 * crabbc.x - fb2 * crbccd.x, fb1 * crabbc.y - fb2 * crbccd.y,
                  fb1 * crabbc.z - fb2 * crbccd.z, fs);
        const double gab = fa + fb1;
        const double gcd = fb2 + fd;
        v.force64(ka, gcd * crbccd.x - gab * crabbc.x, gcd * crbccd.y - gab * crabbc.y,
                  gcd * crbccd.z - gab * crabbc.z, fs);
      }
    }
    if (ENERGY) {
      v.energy64(k, kProperDihedral, e_prop, es);
      v.energy64(k, kImproperDihedral, e_impr, es);
      v.energy64(k, kElec14, e_el14, es);
      v.energy64(k, kVdw14, e_lj14, es);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Tile walks
// ------------------------------------------------------------------------------------------------
struct TileInfo {
  int k;        // unit molecule
  int ibase;    // first slot of block I
  int jbase;    // first slot of block J
  int ni;       // valid atoms in block I
  int nj;       // valid atoms in block J
  bool diag;
  int local;    // tile index within the molecule
};

__device__ __forceinline__ TileInfo tileInfo(const UnitSmem &s, int nsys_u, int t) {
  TileInfo ti;
  ti.k = findOwner(s.tile0, nsys_u, t);
  ti.local = t - s.tile0[ti.k];
  int I, J;
  tileCoordinates(ti.local, &I, &J);
  const int n = s.natom[ti.k];
  ti.ibase = s.slot0[ti.k] + I * kTile;
  ti.jbase = s.slot0[ti.k] + J * kTile;
  ti.ni = min(kTile, n - I * kTile);
  ti.nj = min(kTile, n - J * kTile);
  ti.diag = (I == J);
  return ti;
}

// Run one tile: p.pair(jslot, jl) for every pair of the tile (once each) and p.rotate() after
// every step.  Padding slots hold parameters that make every contribution to a real atom exactly
// zero (no charge, zero screened radius and dE/dR, masked Lennard-Jones, far-away coordinates),
// so partial tiles run the same branch-free loop; only the last step of a diagonal tile, where
// lanes l and l + 16 would meet the same pair, runs on half the lanes.
//
// tileFlush(p) runs after every eighth step and at the end of the tile: passes that sum energies
// in FP32 move their partial sums into integer accumulators there, so no FP32 running sum spans
// more than eight pairs (the generic overload does nothing).
template <class P>
__device__ __forceinline__ void tileFlush(P &) {}

template <class P>
__device__ __forceinline__ void walkTile(P &p, const TileInfo &ti, int lane) {
  if (!ti.diag) {
#pragma unroll 1
    for (int k0 = 0; k0 < kTile; k0 += 8) {
#pragma unroll 2
      for (int k = k0; k < k0 + 8; k++) {
        const int jl = (lane + k) & 31;
        p.pair(ti.jbase + jl, jl);
        p.rotate(lane);
      }
      tileFlush(p);
    }
  }
  else {
#pragma unroll 1
    for (int k = 1; k < 16; k++) {
      const int jl = (lane + k) & 31;
      p.pair(ti.jbase + jl, jl);
      p.rotate(lane);
      if (k == 8) {
        tileFlush(p);
      }
    }
    if (lane < 16) {
      p.pair(ti.jbase + lane + 16, lane + 16);
    }
    p.rotate(lane);
    tileFlush(p);
  }
}

// Walk a tile two pairs per lane per step: an off-diagonal tile in 16 steps pairing j = l + k
// with j = l + k + 16, a diagonal tile in 8 steps pairing j = l + k with j = l + k + 8 (the
// second pair of the last step on half the lanes: w2 = 0 elsewhere).  Each of the two j streams
// carries its own traveling accumulators; p.merge() folds the second into the first, after which
// lane l holds those of block J's atom (l + 16) mod 32 (off-diagonal) or (l + 9) mod 32.
template <class P>
__device__ __forceinline__ void walkTile2(P &p, const TileInfo &ti, int lane) {
  if (!ti.diag) {
#pragma unroll 2
    for (int k = 0; k < 16; k++) {
      const int j1 = (lane + k) & 31;
      const int j2 = (lane + k + 16) & 31;
      p.pair2(ti.jbase + j1, j1, ti.jbase + j2, j2, 1.0f);
      p.rotate2(lane);
    }
    p.merge((lane + 16) & 31);
  }
  else {
#pragma unroll 1
    for (int k = 1; k <= 8; k++) {
      const int j1 = (lane + k) & 31;
      const int j2 = (lane + k + 8) & 31;
      p.pair2(ti.jbase + j1, j1, ti.jbase + j2, j2, (k == 8 && lane >= 16) ? 0.0f : 1.0f);
      p.rotate2(lane);
    }
    p.merge((lane + 24) & 31);
  }
}

__device__ __forceinline__ int traveledAtom2(const TileInfo &ti, int lane) {
  return (lane + (ti.diag ? 9 : 16)) & 31;
}

// Lane that holds block J's atom jl's traveling accumulator once the walk is over
__device__ __forceinline__ int traveledAtom(const TileInfo &ti, int lane) {
  return (lane + (ti.diag ? 17 : 32)) & 31;
}

// GB pass 1, two pairs per lane per step: psi_i -= H(r, rho_i, s_j rho_j) and
// psi_j -= H(r, rho_j, s_i rho_i)
template <bool NECK = false>
struct RadiiPass2 {
  const UnitSmem &s;
  NeckGb neck;
  float4 ai, bi;
  int ni;           // neck index of atom i
  float2 psi_i2;    // i-side sums of the two pair streams
  float2 psi_j;     // traveling j-side sums: x for stream 1, y for stream 2
  float psi_i, psi_j1;
  __device__ RadiiPass2(const UnitSmem &s_in, const DevSynthesis &d) : s(s_in), neck(d) {}
  __device__ __forceinline__ void begin(int islot) {
    ai = s.pa[islot];
    bi = s.pb[islot];
    if (NECK) {
      ni = s.neck[islot];
    }
    psi_i2 = f2(0.0f);
    psi_j = f2(0.0f);
  }
  __device__ __forceinline__ void pair2(int js1, int, int js2, int, float w2) {
    const float4 aj1 = s.pa[js1];
    const float4 bj1 = s.pb[js1];
    const float4 aj2 = s.pa[js2];
    const float4 bj2 = s.pb[js2];
    const float2 dx = add2(sub2(f2(aj1.x, aj2.x), f2(ai.x)), sub2(f2(bj1.x, bj2.x), f2(bi.x)));
    const float2 dy = add2(sub2(f2(aj1.y, aj2.y), f2(ai.y)), sub2(f2(bj1.y, bj2.y), f2(bi.y)));
    const float2 dz = add2(sub2(f2(aj1.z, aj2.z), f2(ai.z)), sub2(f2(bj1.z, bj2.z), f2(bi.z)));
    const float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    const float2 invr = f2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 r = mul2(r2, invr);
    float2 hi = hctIntegral2(r, r2, invr, f2(bi.w), f2(aj1.w, aj2.w));
    float2 hj = hctIntegral2(r, r2, invr, f2(bj1.w, bj2.w), f2(ai.w));
    if (NECK) {
      if (r.x < bi.w + bj1.w + neck.reach) {
        const int nj = s.neck[js1];
        hi.x += neck.integral(ni, nj, r.x);
        hj.x += neck.integral(nj, ni, r.x);
      }
      if (r.y < bi.w + bj2.w + neck.reach) {
        const int nj = s.neck[js2];
        hi.y += neck.integral(ni, nj, r.y);
        hj.y += neck.integral(nj, ni, r.y);
      }
    }
    const float2 wneg = f2(-1.0f, -w2);
    psi_i2 = fma2(hi, wneg, psi_i2);
    psi_j = fma2(hj, wneg, psi_j);
  }
  __device__ __forceinline__ void rotate2(int lane) {
    psi_j.x = __shfl_sync(kFullMask, psi_j.x, (lane + 1) & 31);
    psi_j.y = __shfl_sync(kFullMask, psi_j.y, (lane + 1) & 31);
  }
  __device__ __forceinline__ void merge(int src) {
    psi_i = psi_i2.x + psi_i2.y;
    psi_j1 = psi_j.x + __shfl_sync(kFullMask, psi_j.y, src);
  }
};

// Pass 2: Coulomb + Lennard-Jones on non-excluded pairs and the GB pair terms; with CLASH, the
// Coulomb and Lennard-Jones terms of a molecule given a clash distance or ratio take softened
// cores (the uniform branch is per tile: a tile belongs to one molecule)
template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH = false>
struct PairPass {
  const UnitSmem &s;
  float kk, inv_diel;
  bool salt;
  float4 ai, bi;
  float inv4ri;     // 1 / (4 R_i)
  int code_i;
  unsigned mask;
  bool soft;        // softened cores on this tile
  float clash_d, clash_r;
  float2 qcore;
  float fxi, fyi, fzi, dei, fxj, fyj, fzj, dej;
  float e_elec, e_vdw, e_gb;        // FP32 sums of at most eight pairs (see tileFlush)
  double t_elec, t_vdw, t_gb;       // this lane's FP64 sums over the tile (see tileEnergy)
  __device__ PairPass(const UnitSmem &s_in, float kappa, float inv_dielectric) :
      s(s_in), kk(-kappa * kGbKscale), inv_diel(inv_dielectric), salt(kappa > 0.0f) {}
  __device__ __forceinline__ void flush() {
    if (ENERGY) {
      t_elec += static_cast<double>(e_elec);
      t_vdw += static_cast<double>(e_vdw);
      t_gb += static_cast<double>(e_gb);
      e_elec = e_vdw = e_gb = 0.0f;
    }
  }
  __device__ __forceinline__ void begin(int islot, unsigned mask_in,
                                        float2 clash = make_float2(0.0f, 0.0f)) {
    ai = s.pa[islot];
    bi = s.pb[islot];
    inv4ri = 0.25f * s.gbv[islot].x;
    code_i = __float_as_int(s.prm[islot].y) & 0xffff;
    mask = mask_in;
    if (CLASH) {
      clash_d = clash.x;
      clash_r = clash.y;
      soft = (clash.x > 0.0f || clash.y > 0.0f);
      qcore = quadraticCore(clash.x);
    }
    fxi = fyi = fzi = dei = 0.0f;
    fxj = fyj = fzj = dej = 0.0f;
    e_elec = e_vdw = e_gb = 0.0f;
    t_elec = t_vdw = t_gb = 0.0;
  }
  __device__ __forceinline__ void pair(int jslot, int jl) {
    const float4 aj = s.pa[jslot];
    const float4 bj = s.pb[jslot];
    const float2 gj = s.gbv[jslot];    // pass 2: 1 / effective radius, Lennard-Jones code bits
    const float hx = aj.x - ai.x, hy = aj.y - ai.y, hz = aj.z - ai.z;
    const float lx = bj.x - bi.x, ly = bj.y - bi.y, lz = bj.z - bi.z;
    const float3 dv = make_float3(hx + lx, hy + ly, hz + lz);
    const float r2 = fmaf(dv.x, dv.x, fmaf(dv.y, dv.y, dv.z * dv.z));
    const float qiqj_all = ai.w * aj.w;
    float fmag = 0.0f;
    if (NB) {
      // excluded and padding pairs take the same path with zero parameters
      const float incl = ((mask >> jl) & 1u) ? 0.0f : 1.0f;
      // 1/r from rsqrt with one Newton step (Coulomb), and 1/r^2 as its own reciprocal: r^-6
      // and r^-12 multiply the relative error of 1/r^2 by 3 and 6, so squaring 1/r (twice its
      // error) would double the rounding of the repulsive wall, and the Newton step of 1/r^2
      // takes the exact r^2 = r2 + 2 (dx ex + dy ey + dz ez) + O(e^2), the e the separations'
      // recovered rounding errors (separationError): without it the Lennard-Jones energy of a
      // molecule with close contacts errs by up to 1.5e-6 of the root-sum-square of its pair
      // terms.  r2 >= 256 on padding slots, never zero.
      float invr = rsqrtf(r2);
      invr = invr * fmaf(-0.5f * r2 * invr, invr, 1.5f);
      const float r2c = fmaf(dv.x, separationError(hx, lx, dv.x),
                             fmaf(dv.y, separationError(hy, ly, dv.y),
                                  dv.z * separationError(hz, lz, dv.z)));
      float invr2 = __fdividef(1.0f, r2);
      invr2 = fmaf(invr2, fmaf(-2.0f * r2c, invr2, fmaf(-r2, invr2, 1.0f)), invr2);
      const float invr6 = invr2 * invr2 * invr2;
      float2 ab = s.lj[code_i + (__float_as_int(gj.y) >> 16)];
      ab.x *= incl;
      ab.y *= incl;
      const float qiqj = qiqj_all * incl;
      if (CLASH && soft) {
        fmag = softCorePair(r2 * invr, invr, qiqj, ab.x, ab.y, clash_d, qcore, clash_r, &e_elec,
                            &e_vdw);
      }
      else {
        if (ENERGY) {
          e_elec = __fadd_rn(e_elec, __fmul_rn(qiqj, invr));
          e_vdw = __fadd_rn(e_vdw, __fmul_rn(__fsub_rn(__fmul_rn(ab.x, invr6), ab.y), invr6));
        }
        if (FORCE) {
          fmag = -(qiqj * invr * invr2) + (6.0f * ab.y - 12.0f * ab.x * invr6) * invr6 * invr2;
        }
      }
    }
    if (GB) {
      const float qiqj = qiqj_all;
      const float ijb = bi.w * bj.w;
      const float efac = __expf(-r2 * inv4ri * gj.x);
      const float fgbi = rsqrtf(fmaf(ijb, efac, r2));
      float expmkf, fgbk;
      if (salt) {
        fgbk = __fdividef(kk, fgbi);
        expmkf = __expf(fgbk) * inv_diel;
      }
      else {
        fgbk = 0.0f;
        expmkf = inv_diel;
      }
      const float dielfac = 1.0f - expmkf;
      if (ENERGY) {
        e_gb = __fsub_rn(e_gb, __fmul_rn(__fmul_rn(qiqj, dielfac), fgbi));
      }
      if (FORCE) {
        const float temp4 = fgbi * fgbi * fgbi;
        const float temp6 = qiqj * temp4 * fmaf(fgbk, expmkf, dielfac);
        fmag += temp6 * fmaf(-0.25f, efac, 1.0f);
        const float temp5 = 0.5f * efac * temp6 * fmaf(0.25f, r2, ijb);
        dei = fmaf(bi.w, temp5, dei);
        dej = fmaf(bj.w, temp5, dej);
      }
    }
    if (FORCE) {
      fxi = fmaf(fmag, dv.x, fxi);
      fyi = fmaf(fmag, dv.y, fyi);
      fzi = fmaf(fmag, dv.z, fzi);
      fxj = fmaf(-fmag, dv.x, fxj);
      fyj = fmaf(-fmag, dv.y, fyj);
      fzj = fmaf(-fmag, dv.z, fzj);
    }
  }
  __device__ __forceinline__ void rotate(int lane) {
    if (FORCE) {
      const int src = (lane + 1) & 31;
      fxj = __shfl_sync(kFullMask, fxj, src);
      fyj = __shfl_sync(kFullMask, fyj, src);
      fzj = __shfl_sync(kFullMask, fzj, src);
      if (GB) {
        dej = __shfl_sync(kFullMask, dej, src);
      }
    }
  }
};

template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH>
__device__ __forceinline__ void tileFlush(PairPass<FORCE, ENERGY, NB, GB, CLASH> &p) {
  p.flush();
}

// Pass 3: radius chain-rule forces
template <bool NECK = false>
struct DerivPass {
  const UnitSmem &s;
  NeckGb neck;
  float4 ai, bi;
  int ni;
  float de_i;
  float fxi, fyi, fzi, fxj, fyj, fzj;
  __device__ DerivPass(const UnitSmem &s_in, const DevSynthesis &d) : s(s_in), neck(d) {}
  __device__ __forceinline__ void begin(int islot) {
    ai = s.pa[islot];
    bi = s.pb[islot];
    if (NECK) {
      ni = s.neck[islot];
    }
    de_i = s.gbv[islot].y;
    fxi = fyi = fzi = 0.0f;
    fxj = fyj = fzj = 0.0f;
  }
  __device__ __forceinline__ void pair(int jslot, int) {
    const float4 aj = s.pa[jslot];
    const float4 bj = s.pb[jslot];
    const float de_j = s.gbv[jslot].y;
    const float3 dv = pairDelta(ai, bi, aj, bj);
    const float r2 = fmaf(dv.x, dv.x, fmaf(dv.y, dv.y, dv.z * dv.z));
    const float invr = rsqrtf(r2);
    const float r = r2 * invr;
    // scalar forms: on the long chains of the tiled path nearly every pair is far, and the
    // packed pair form measured slower there
    float fmag = hctDerivative(r, r2, invr, bi.w, aj.w) * de_i +
                 hctDerivative(r, r2, invr, bj.w, ai.w) * de_j;
    if (NECK && r < bi.w + bj.w + neck.reach) {
      const int nj = s.neck[jslot];
      float dij, dji;
      neck.both(ni, nj, r, invr, &dij);
      neck.both(nj, ni, r, invr, &dji);
      fmag += dij * de_i + dji * de_j;
    }
    fxi = fmaf(-fmag, dv.x, fxi);
    fyi = fmaf(-fmag, dv.y, fyi);
    fzi = fmaf(-fmag, dv.z, fzi);
    fxj = fmaf(fmag, dv.x, fxj);
    fyj = fmaf(fmag, dv.y, fyj);
    fzj = fmaf(fmag, dv.z, fzj);
  }
  __device__ __forceinline__ void rotate(int lane) {
    const int src = (lane + 1) & 31;
    fxj = __shfl_sync(kFullMask, fxj, src);
    fyj = __shfl_sync(kFullMask, fyj, src);
    fzj = __shfl_sync(kFullMask, fzj, src);
  }
};

// GB pass 1 of a force evaluation: psi_i -= H(r, rho_i, s_j rho_j), psi_j -= H(r, rho_j,
// s_i rho_i), and the radial derivatives of both terms stored for pass 3 (one float2 per lane
// and step of the tile walk, so the stores of a step are one coalesced 256-byte line)
template <bool NECK = false>
struct RadiiDerivPass {
  const UnitSmem &s;
  NeckGb neck;
  float4 ai, bi;
  int ni;
  float psi_i, psi_j;   // i-side sum, traveling j-side sum
  float2* out;          // this lane's entry for the current step
  __device__ RadiiDerivPass(const UnitSmem &s_in, const DevSynthesis &d) : s(s_in), neck(d) {}
  __device__ __forceinline__ void begin(int islot, float2* tile_out) {
    ai = s.pa[islot];
    bi = s.pb[islot];
    if (NECK) {
      ni = s.neck[islot];
    }
    psi_i = 0.0f;
    psi_j = 0.0f;
    out = tile_out;
  }
  __device__ __forceinline__ void pair(int jslot, int) {
    const float4 aj = s.pa[jslot];
    const float4 bj = s.pb[jslot];
    const float2 dxy = add2(sub2(f2(aj.x, aj.y), f2(ai.x, ai.y)),
                            sub2(f2(bj.x, bj.y), f2(bi.x, bi.y)));
    const float dz = (aj.z - ai.z) + (bj.z - bi.z);
    const float r2 = fmaf(dxy.x, dxy.x, fmaf(dxy.y, dxy.y, dz * dz));
    const float invr = rsqrtf(r2);
    const float r = r2 * invr;
    float2 h, hd;
    hctBoth2(r, r2, invr, f2(bi.w, bj.w), f2(aj.w, ai.w), &h, &hd);
    if (NECK && r < bi.w + bj.w + neck.reach) {
      const int nj = s.neck[jslot];
      float dij, dji;
      h.x += neck.both(ni, nj, r, invr, &dij);
      h.y += neck.both(nj, ni, r, invr, &dji);
      hd.x += dij;
      hd.y += dji;
    }
    psi_i -= h.x;
    psi_j -= h.y;
    __stcg(out, hd);
  }
  __device__ __forceinline__ void rotate(int lane) {
    psi_j = __shfl_sync(kFullMask, psi_j, (lane + 1) & 31);
    out += 32;
  }
};

// Pass 3 from the stored derivatives: the force of a pair is (hd_i dE/dR_i + hd_j dE/dR_j) times
// the separation, with no transcendental left to evaluate
struct DerivStoredPass {
  const UnitSmem &s;
  float4 ai, bi;
  float de_i;
  float2 fxyi, fxyj;
  float fzi, fzj;
  const float2* in;
  __device__ DerivStoredPass(const UnitSmem &s_in) : s(s_in) {}
  __device__ __forceinline__ void begin(int islot, const float2* tile_in) {
    ai = s.pa[islot];
    bi = s.pb[islot];
    de_i = s.gbv[islot].y;
    fxyi = fxyj = f2(0.0f);
    fzi = fzj = 0.0f;
    in = tile_in;
  }
  __device__ __forceinline__ void pair(int jslot, int) {
    const float2 hd = __ldcs(in);
    const float4 aj = s.pa[jslot];
    const float4 bj = s.pb[jslot];
    const float de_j = s.gbv[jslot].y;
    const float2 dxy = add2(sub2(f2(aj.x, aj.y), f2(ai.x, ai.y)),
                            sub2(f2(bj.x, bj.y), f2(bi.x, bi.y)));
    const float dz = (aj.z - ai.z) + (bj.z - bi.z);
    const float fmag = fmaf(hd.y, de_j, hd.x * de_i);
    fxyi = fma2(f2(-fmag), dxy, fxyi);
    fzi = fmaf(-fmag, dz, fzi);
    fxyj = fma2(f2(fmag), dxy, fxyj);
    fzj = fmaf(fmag, dz, fzj);
  }
  __device__ __forceinline__ void rotate(int lane) {
    const int src = (lane + 1) & 31;
    fxyj.x = __shfl_sync(kFullMask, fxyj.x, src);
    fxyj.y = __shfl_sync(kFullMask, fxyj.y, src);
    fzj = __shfl_sync(kFullMask, fzj, src);
    in += 32;
  }
};

// Entry of lane 0, step 0 of tile t of a unit whose tiles start at tile_base in the store
__device__ __forceinline__ size_t pairDerivOffset(int tile_base, int t) {
  return static_cast<size_t>(tile_base + t) * kPairDerivPerTile;
}

template <bool STORE, bool NECK>
__device__ void gbRadiiTiles(const DevSynthesis &d, const UnitSmem &s, int nsys_u, int ntiles,
                             int tile_base, int first, int stride) {
  const int lane = threadIdx.x & 31;
  const float ps = static_cast<float>(1 << kPsiBits);
  if (STORE) {
    RadiiDerivPass<NECK> p(s, d);
    for (int t = first; t < ntiles; t += stride) {
      const TileInfo ti = tileInfo(s, nsys_u, t);
      p.begin(ti.ibase + lane, d.pair_deriv + pairDerivOffset(tile_base, t) + lane);
      walkTile(p, ti, lane);
      if (lane < ti.ni) {
        atomicAddInt63(p.psi_i * ps, &s.psi[ti.ibase + lane], &s.psio[ti.ibase + lane]);
      }
      const int jl = traveledAtom(ti, lane);
      if (jl < ti.nj) {
        atomicAddInt63(p.psi_j * ps, &s.psi[ti.jbase + jl], &s.psio[ti.jbase + jl]);
      }
    }
    return;
  }
  RadiiPass2<NECK> p(s, d);
  for (int t = first; t < ntiles; t += stride) {
    const TileInfo ti = tileInfo(s, nsys_u, t);
    p.begin(ti.ibase + lane);
    walkTile2(p, ti, lane);
    if (lane < ti.ni) {
      atomicAddInt63(p.psi_i * ps, &s.psi[ti.ibase + lane], &s.psio[ti.ibase + lane]);
    }
    const int jl = traveledAtom2(ti, lane);
    if (jl < ti.nj) {
      atomicAddInt63(p.psi_j1 * ps, &s.psi[ti.jbase + jl], &s.psio[ti.jbase + jl]);
    }
  }
}

template <bool FORCE, bool ENERGY, bool NB, bool GB, bool CLASH = false>
__device__ void pairTiles(const DevSynthesis &d, const UnitSmem &s, int nsys_u, int ntiles,
                          int first, int stride) {
  const int lane = threadIdx.x & 31;
  const float fs = d.frc_scale;
  const float es = d.nrg_scale;
  const float ds = static_cast<float>(1 << kDeijdaBits);
  PairPass<FORCE, ENERGY, NB, GB, CLASH> p(s, d.kappa, d.inv_dielectric);
  // a molecule's energies over this warp's tiles, each tile rounded to the output grid
  // (tileEnergy), the same value in every lane
  long long acc_elec = 0, acc_vdw = 0, acc_gb = 0;
  int acc_k = -1;
  auto commit = [&]() {
    if (lane == 0 && acc_k >= 0) {
      if (NB) {
        atomicAdd(&s.nrg[acc_k * kNrgStride + kElec], static_cast<unsigned long long>(acc_elec));
        atomicAdd(&s.nrg[acc_k * kNrgStride + kVdw], static_cast<unsigned long long>(acc_vdw));
      }
      if (GB) {
        atomicAdd(&s.nrg[acc_k * kNrgStride + kGb], static_cast<unsigned long long>(acc_gb));
      }
    }
    acc_elec = acc_vdw = acc_gb = 0;
  };
  for (int t = first; t < ntiles; t += stride) {
    const TileInfo ti = tileInfo(s, nsys_u, t);
    if (ENERGY && ti.k != acc_k) {
      commit();
      acc_k = ti.k;
    }
    unsigned mask = 0u;
    if (NB) {
      const int midx = d.tile_mask_idx[d.tile_start[s.sys[ti.k]] + ti.local];
      if (midx != 0) {
        mask = __ldg(&d.mask_pool[static_cast<size_t>(midx) * 32 + lane]);
      }
    }
    p.begin(ti.ibase + lane, mask, CLASH ? s.clash[ti.k] : make_float2(0.0f, 0.0f));
    walkTile(p, ti, lane);
    if (FORCE) {
      if (lane < ti.ni) {
        const int is = ti.ibase + lane;
        addForce(s, is, p.fxi, p.fyi, p.fzi, fs);
        if (GB) {
          atomicAddInt63(p.dei * ds, &s.de[is], &s.deo[is]);
        }
      }
      const int jl = traveledAtom(ti, lane);
      if (jl < ti.nj) {
        const int js = ti.jbase + jl;
        addForce(s, js, p.fxj, p.fyj, p.fzj, fs);
        if (GB) {
          atomicAddInt63(p.dej * ds, &s.de[js], &s.deo[js]);
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
  }
  if (ENERGY) {
    commit();
  }
}

__device__ void gbDerivativeTiles(const DevSynthesis &d, const UnitSmem &s, int nsys_u,
                                  int ntiles, int tile_base, int first, int stride) {
  const int lane = threadIdx.x & 31;
  const float fs = d.frc_scale;
  DerivStoredPass p(s);
  for (int t = first; t < ntiles; t += stride) {
    const TileInfo ti = tileInfo(s, nsys_u, t);
    p.begin(ti.ibase + lane, d.pair_deriv + pairDerivOffset(tile_base, t) + lane);
    walkTile(p, ti, lane);
    if (lane < ti.ni) {
      addForce(s, ti.ibase + lane, p.fxyi.x, p.fxyi.y, p.fzi, fs);
    }
    const int jl = traveledAtom(ti, lane);
    if (jl < ti.nj) {
      addForce(s, ti.jbase + jl, p.fxyj.x, p.fxyj.y, p.fzj, fs);
    }
  }
}
// ------------------------------------------------------------------------------------------------
// Per-atom GB steps between the pair passes (nonbonded_potential.tpp:730-805, 982-1021)
// ------------------------------------------------------------------------------------------------
// Effective radius of atom gi from its descreening sum psi (HCT, or OBC / OBC-II)
// Effective GB radius of an atom from its descreening sum psi, in FP64 with the FP64
// parameters: the OBC form 1 / (1 / rho - tanh(...) / r) cancels for buried atoms, where tanh
// nears 1 and 1 / rho - 1 / r is a small difference, and FP32 there loses the 1e-6 relative
// accuracy of the GB energy on compact proteins.  One evaluation per atom, so FP64 costs
// nothing measurable.
__device__ __forceinline__ float effectiveRadius(const DevSynthesis &d, int gi, double psi) {
  const double4 p = d.gb_radius64[gi];   // rho, intrinsic radius, alpha, beta
  double egbi;
  if (d.igb == 1) {
    egbi = 1.0 / (1.0 / p.x + psi);
    if (egbi < 0.0) egbi = 30.0;
  }
  else {
    const double fipsi = psi * (-p.x);
    egbi = 1.0 / (1.0 / p.x - tanh((p.z - p.w * fipsi + d.gb_gamma64[gi] * fipsi * fipsi) *
                                   fipsi) / p.y);
  }
  return static_cast<float>(egbi);
}

// GB self energy of a charge q (scaled by sqrt of the Coulomb constant) with effective radius
// egbi; *self_de receives its dE/dR contribution
__device__ __forceinline__ float gbSelfTerm(const DevSynthesis &d, float q, float egbi,
                                            float* self_de) {
  const float expmkf = ((d.kappa > 0.0f) ? expf(-kGbKscale * d.kappa * egbi) : 1.0f) *
                       d.inv_dielectric;
  const float dielfac = 1.0f - expmkf;
  const float atmq2h = 0.5f * q * q;
  const float atmqd2h = atmq2h * dielfac;
  *self_de = atmqd2h - kGbKscale * d.kappa * atmq2h * expmkf * egbi;
  return -__fdiv_rn(atmqd2h, egbi);
}

// OBC chain-rule factor dR/dpsi-type prefactor applied to the summed dE/dR
// OBC chain-rule factor (the dR/dpsi-type prefactor applied to the summed dE/dR), in FP64 for
// the same reason: 1 - tanh^2 cancels where tanh nears 1
__device__ __forceinline__ float obcChainFactor(const DevSynthesis &d, int gi, double psi) {
  const double4 p = d.gb_radius64[gi];
  const double fipsi = psi * (-p.x);
  const double ga = d.gb_gamma64[gi];
  const double thi = tanh((p.z - (p.w - ga * fipsi) * fipsi) * fipsi);
  return static_cast<float>((p.z - (2.0 * p.w - 3.0 * ga * fipsi) * fipsi) * (1.0 - thi * thi) *
                            p.x / p.y);
}

// ------------------------------------------------------------------------------------------------
// Work-unit staging and the staged evaluation, shared by the evaluation and minimization kernels
// ------------------------------------------------------------------------------------------------
struct UnitShape {
  int nsys;       // molecules in the unit
  int nslots;     // atom slots (sum of the molecules' sizes padded to 32)
  int ntiles;     // 32 x 32 tiles of the molecules' lower triangles
  int tile_base;  // first tile of the unit in the pair-derivative store
};

// Molecule table, prefix sums and Lennard-Jones tables of unit u.  Returns false (after setting
// bit 0 of the status word) when the unit does not fit the launch's shared-memory carve-out; the
// caller then skips the unit.  Ends with a barrier.
template <class Team>
__device__ bool stageUnitTables(const DevSynthesis &d, const UnitSmem &s, int u, int max_lj,
                                UnitShape* shape, const Team &team, int max_sys = kMaxUnitSystems) {
  const int4 desc = d.unit_desc[u];
  const int nsys_u = desc.y;
  shape->nsys = nsys_u;
  shape->nslots = desc.z;
  shape->ntiles = desc.w;
  if (nsys_u > max_sys) {
    if (team.rank() == 0) {
      atomicOr(d.status, 1);
    }
    return false;
  }
  // the unit's molecule table, precomputed on the host: one coalesced load per field
  const int* meta = d.unit_meta + static_cast<size_t>(desc.x) * kUnitMetaFields;
  shape->tile_base = meta[nsys_u * kUnitMetaFields];
  for (int e = team.rank(); e < (nsys_u + 1) * kUnitMetaFields; e += team.size()) {
    const int k = e / kUnitMetaFields;
    const int v = meta[e];
    switch (e % kUnitMetaFields) {
      case 0: if (k < nsys_u) s.sys[k] = v; break;
      case 1: if (k < nsys_u) s.natom[k] = v; break;
      case 2: if (k < nsys_u) s.slot0[k] = v; break;
      case 3: s.tile0[k] = v; break;
      case 4: s.ljbase[k] = v; break;
      case 5: s.bchunk0[k] = v; break;
      case 6: s.achunk0[k] = v; break;
      default: s.dchunk0[k] = v; break;
    }
  }
  team.sync();
  if (desc.z > d.max_unit_slots || s.ljbase[nsys_u] > max_lj || nsys_u > max_sys) {
    if (team.rank() == 0) {
      atomicOr(d.status, 1);
    }
    return false;   // reported through the status word; nothing in the unit is touched
  }
  // Lennard-Jones tables (standard then 1-4) of every molecule, all entries in parallel
  for (int e = team.rank(); e < s.ljbase[nsys_u]; e += team.size()) {
    const int k = findOwner(s.ljbase, nsys_u, e);
    const int sysid = s.sys[k];
    const int nt = d.lj_ntypes[sysid];
    const int rel = e - s.ljbase[k];
    const int src = d.lj_start[sysid] + (rel < nt * nt ? rel : rel - nt * nt);
    s.lj[e] = (rel < nt * nt) ? d.ljab[src] : d.ljab14[src];
  }
  team.sync();
  return true;
}

// Static per-slot parameters of an atom (a < natom) or of a padding slot: charge, Lennard-Jones
// code, rho, s * rho.  A padding slot has no charge, zero screened radius and a masked
// Lennard-Jones row, so every pair term it enters is exactly zero for the real atom.
__device__ __forceinline__ float4 slotParameters(const DevSynthesis &d, const UnitSmem &s, int k,
                                                 int a) {
  if (a < s.natom[k]) {
    const int sysid = s.sys[k];
    const int gi = d.atom_start[sysid] + a;
    const int nt = d.lj_ntypes[sysid];
    const int ty = d.lj_idx[gi];
    return make_float4(d.charge[gi], __int_as_float((s.ljbase[k] + ty * nt) | (ty << 16)),
                       d.rho[gi], d.srho[gi]);
  }
  return make_float4(0.0f, __int_as_float(s.ljbase[k]), 1.0f, 0.0f);
}

// Neck GB table index of slot a of unit molecule k (0 for padding or other GB models)
__device__ __forceinline__ int slotNeck(const DevSynthesis &d, const UnitSmem &s, int k, int a) {
  return (d.neck_size > 0 && a < s.natom[k]) ? d.neck_idx[d.atom_start[s.sys[k]] + a] : 0;
}

// Place an atom (fixed-point coordinates c, real = true) or a padding slot (far from everything:
// 16 A apart along x beyond 5000 A) and clear its accumulators for a new evaluation
__device__ __forceinline__ void placeSlot(const DevSynthesis &d, const UnitSmem &s, int slot,
                                          bool real, long long cx, long long cy, long long cz) {
  const float4 prm = s.prm[slot];
  float4 pa, pb;
  if (real) {
    splitCoordinate(static_cast<double>(cx) * d.inv_gpos_scale, &pa.x, &pb.x);
    splitCoordinate(static_cast<double>(cy) * d.inv_gpos_scale, &pa.y, &pb.y);
    splitCoordinate(static_cast<double>(cz) * d.inv_gpos_scale, &pa.z, &pb.z);
  }
  else {
    pa = make_float4(5000.0f + 16.0f * static_cast<float>(slot), 0.0f, 0.0f, 0.0f);
    pb = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  pa.w = prm.w;   // pass 1 payload: s * rho
  pb.w = prm.z;   //                 rho
  s.pa[slot] = pa;
  s.pb[slot] = pb;
  s.gbv[slot] = make_float2(1.0f, 0.0f);
  s.fx[slot] = 0;
  s.fy[slot] = 0;
  s.fz[slot] = 0;
  s.fxo[slot] = 0;
  s.fyo[slot] = 0;
  s.fzo[slot] = 0;
  s.psi[slot] = 0;
  s.psio[slot] = 0;
  s.de[slot] = 0;
  s.deo[slot] = 0;
}

// All requested terms of a staged unit: coordinates, parameters and cleared accumulators in
// shared memory on entry (and a barrier since); forces in s.fx.. and per-molecule energies in
// s.nrg on exit, after a barrier.  WS: also write the GB workspace (psi, effective radii, dE/dR)
// to global memory.  CLASH: Coulomb and Lennard-Jones pairs, 1-4 pairs included, take the
// softened cores of s.clash (per unit molecule, zero for none, set before that barrier).  NECK:
// the neck GB term (s.neck holds the slots' neck indices).
template <bool FORCE, bool ENERGY, int TERMS, bool WS, bool CLASH = false, bool NECK = false,
          class Team>
__device__ void evaluateStaged(const DevSynthesis &d, const UnitSmem &s, const UnitShape &us,
                               const Team &team) {
  constexpr bool VALE = (TERMS & 1) != 0;
  constexpr bool NB = (TERMS & 2) != 0;
  const bool gb = ((TERMS & 4) != 0) && (d.igb != 0);
  const int nsys_u = us.nsys;
  const int nslots = us.nslots;
  const int ntiles = us.ntiles;

  // valence terms and GB pass 1 touch disjoint accumulators: no barrier between them
  if (VALE) {
    valenceTerms<FORCE, ENERGY, SmemValence, CLASH>(d, SmemValence(s, team.warp(), team.warps()),
                                                    nsys_u);
    if (!gb) {
      team.sync();
    }
  }
  if (gb) {
    gbRadiiTiles<FORCE, NECK>(d, s, nsys_u, ntiles, us.tile_base, team.warp(), team.warps());
    team.sync();
    // effective radii, self terms (nonbonded_potential.tpp:730-805); a warp's 32 slots
    // belong to one molecule, so the self energies reduce across the warp
    const float inv_ps = 1.0f / static_cast<float>(1 << kPsiBits);
    const float ds = static_cast<float>(1 << kDeijdaBits);
    for (int slot = team.rank(); slot < nslots; slot += team.size()) {
      const int k = findOwner(s.slot0, nsys_u, slot);
      const int a = slot - s.slot0[k];
      float e_self = 0.0f;
      float4 pa = s.pa[slot];
      float4 pb = s.pb[slot];
      const float4 prm = s.prm[slot];
      float egbi = 1.0f;
      if (a < s.natom[k]) {
        const int gi = d.atom_start[s.sys[k]] + a;
        const double psi = static_cast<double>(int63ToLong(s.psi[slot], s.psio[slot])) *
                           static_cast<double>(inv_ps);
        egbi = effectiveRadius(d, gi, psi);
        float self_de;
        e_self = gbSelfTerm(d, prm.x, egbi, &self_de);
        if (FORCE) {
          atomicAddInt63(self_de * ds, &s.de[slot], &s.deo[slot]);
        }
        if (WS) {
          d.born_radii[gi] = egbi;
          d.psi[gi] = __double2ll_rn(static_cast<double>(psi) * d.psi_out_scale);
          d.psi_ovrf[gi] = 0;
        }
        pa.w = prm.x;   // pass 2 payload: charge
        pb.w = egbi;    //                 effective radius
      }
      else {
        pa.w = 0.0f;
        pb.w = 1.0f;
      }
      s.pa[slot] = pa;
      s.pb[slot] = pb;
      // pass 2 reads a partner's reciprocal radius and Lennard-Jones code with one load
      s.gbv[slot] = make_float2(1.0f / egbi, prm.y);
      if (ENERGY) {
        warpEnergy(s, k, kGb, e_self, d.nrg_scale);
      }
    }
    team.sync();
  }
  else if (NB) {
    // pass 2 payload for Coulomb / Lennard-Jones alone: charge in w1
    for (int slot = team.rank(); slot < nslots; slot += team.size()) {
      float4 pa = s.pa[slot];
      const float4 prm = s.prm[slot];
      pa.w = prm.x;
      s.gbv[slot].y = prm.y;     // the Lennard-Jones code, where pass 2 reads it
      s.pa[slot] = pa;
    }
    team.sync();
  }
  if (NB || gb) {
    if (NB && gb) {
      pairTiles<FORCE, ENERGY, true, true, CLASH>(d, s, nsys_u, ntiles, team.warp(),
                                                  team.warps());
    }
    else if (NB) {
      pairTiles<FORCE, ENERGY, true, false, CLASH>(d, s, nsys_u, ntiles, team.warp(),
                                                   team.warps());
    }
    else {
      pairTiles<FORCE, ENERGY, false, true>(d, s, nsys_u, ntiles, team.warp(), team.warps());
    }
    team.sync();
  }
  if (gb && FORCE) {
    // chain-rule prefactor of the OBC radii (nonbonded_potential.tpp:982-1021), and the
    // pass 3 payloads
    const float inv_ds = 1.0f / static_cast<float>(1 << kDeijdaBits);
    const float inv_ps = 1.0f / static_cast<float>(1 << kPsiBits);
    for (int slot = team.rank(); slot < nslots; slot += team.size()) {
      const int k = findOwner(s.slot0, nsys_u, slot);
      const int a = slot - s.slot0[k];
      const float4 prm = s.prm[slot];
      float4 pa = s.pa[slot];
      float4 pb = s.pb[slot];
      pa.w = prm.w;   // s * rho
      pb.w = prm.z;   // rho
      float sde = 0.0f;
      if (a < s.natom[k]) {
        const int gi = d.atom_start[s.sys[k]] + a;
        sde = static_cast<float>(int63ToLong(s.de[slot], s.deo[slot])) * inv_ds;
        if (d.igb != 1) {
          const double psi = static_cast<double>(int63ToLong(s.psi[slot], s.psio[slot])) *
                             static_cast<double>(inv_ps);
          sde *= obcChainFactor(d, gi, psi);
        }
        if (WS) {
          d.sumdeijda[gi] = __double2ll_rn(static_cast<double>(sde) * d.psi_out_scale);
          d.sumdeijda_ovrf[gi] = 0;
        }
      }
      s.pa[slot] = pa;
      s.pb[slot] = pb;
      s.gbv[slot].y = sde;
    }
    team.sync();
    gbDerivativeTiles(d, s, nsys_u, ntiles, us.tile_base, team.warp(), team.warps());
    team.sync();
  }
}

}  // namespace

}  // namespace sb

#endif