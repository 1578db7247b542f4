// Graph minimizer: the per-system line-search steps between evaluations, one warp per system.
//
// A cycle of the graph minimizer is a fixed sequence of launches captured once as a CUDA graph:
//   clear forces and energies, force + energy evaluation (kEvalFused)
//   kLineStart    energy E0, gg / dgg / |f|^2, convergence, gamma, conjugate direction, its norm,
//                 first trial move (conjugate_gradient.cui:8-140, line_movement.cui:88-126)
//   clear energies, energy evaluation, kLineMove(1): E1, factor 1.04 or 0.8, second trial move
//   clear energies, energy evaluation, kLineMove(2): E2, factor x1.03 or x0.85, third trial move
//   clear energies, energy evaluation, kLineFinish: E3, cubic placement, next move length
// Each evaluation is the batched evaluation kernel at its best launch shape; the steps in between
// are a warp per system with no block-wide barrier.  Per-system sums run over 32-atom chunks in
// a fixed order, so a system's trajectory does not depend on the other systems of the batch.
#include <cuda_runtime.h>

#include "device_kits.h"
#include "fixed_point.cuh"
#include "line_search.cuh"

namespace sb {

namespace {

constexpr int kLineThreads = 256;

__device__ __forceinline__ long long warpSumLong(long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// Total potential energy of a system from its integer energy slots
__device__ __forceinline__ double systemEnergy(const DevSynthesis &d, int sys, int lane) {
  long long v = 0;
  if (lane < kNrgStride) {
    v = static_cast<long long>(d.energies[static_cast<size_t>(sys) * kNrgStride + lane]);
  }
  return static_cast<double>(warpSumLong(v)) / static_cast<double>(d.nrg_scale);
}

__device__ __forceinline__ int firstWarp() {
  return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}

__device__ __forceinline__ int warpStride() { return (gridDim.x * blockDim.x) >> 5; }

// Move every atom of a system by step (fixed-point units per unit of direction); DBL: the FP64
// mode's direction
template <bool DBL>
__device__ __forceinline__ void moveSystem(const DevSynthesis &d, const DevMinimizer &m, int sys,
                                           double step, int lane) {
  if (step == 0.0) {
    return;
  }
  const int natom = d.atom_count[sys];
  const int base = d.atom_start[sys];
  for (int a = lane; a < natom; a += 32) {
    const int gi = base + a;
    if (DBL) {
      m.xcrd[gi] += __double2ll_rn(m.xcg64[gi] * step);
      m.ycrd[gi] += __double2ll_rn(m.ycg64[gi] * step);
      m.zcrd[gi] += __double2ll_rn(m.zcg64[gi] * step);
    }
    else {
      m.xcrd[gi] += __double2ll_rn(static_cast<double>(m.xcg[gi]) * step);
      m.ycrd[gi] += __double2ll_rn(static_cast<double>(m.ycg[gi]) * step);
      m.zcrd[gi] += __double2ll_rn(static_cast<double>(m.zcg[gi]) * step);
    }
  }
}

// Conjugate-gradient step of one system at its line start (conjugate_gradient.cui:8-140):
// energy E0 into the history, gg, dgg and |f|^2 over 32-atom chunks in a fixed order, the RMS
// force and the convergence test, gamma (zero for the first sd_cycles cycles), the new direction
// from the forces and its FP64 norm.  Returns false, with the system marked inactive for the
// cycle, when it has converged or used up its cycles.
template <bool HIST, bool DBL>
__device__ __forceinline__ bool conjugateSystem(const DevSynthesis &d, const DevMinimizer &m,
                                                int sys, double e0, int lane) {
  const double inv_fs = 1.0 / static_cast<double>(d.frc_scale);
  double* line = m.line + static_cast<size_t>(sys) * kLineFields;
  const int cyc = m.cycle[sys];
  if (m.done[sys] || cyc >= m.max_cycles) {
    if (lane == 0) line[kLineAct] = 0.0;
    return false;
  }
    const int natom = d.atom_count[sys];
  const int base = d.atom_start[sys];
  double gg = 0.0, dgg = 0.0, ff = 0.0;
  for (int c = 0; c < natom; c += 32) {
    const int a = c + lane;
    double g = 0.0, dg = 0.0, f2s = 0.0;
    if (a < natom) {
      const int gi = base + a;
      const double fx = int95ToDouble(d.xfrc[gi], d.xfrc_ovrf[gi]);
      const double fy = int95ToDouble(d.yfrc[gi], d.yfrc_ovrf[gi]);
      const double fz = int95ToDouble(d.zfrc[gi], d.zfrc_ovrf[gi]);
      const double px = static_cast<double>(m.xprv[gi]);
      const double py = static_cast<double>(m.yprv[gi]);
      const double pz = static_cast<double>(m.zprv[gi]);
      g = px * px + py * py + pz * pz;
      dg = (fx - px) * fx + (fy - py) * fy + (fz - pz) * fz;
      f2s = fx * fx + fy * fy + fz * fz;
    }
    gg += warpSumDouble(g);
    dgg += warpSumDouble(dg);
    ff += warpSumDouble(f2s);
  }
  gg *= inv_fs * inv_fs;
  dgg *= inv_fs * inv_fs;
  ff *= inv_fs * inv_fs;
  const double rms = sqrt(ff / (3.0 * static_cast<double>(natom)));
  if (lane == 0) {
    m.rms_force[sys] = rms;
    if (HIST && cyc < m.hist_stride) {
      m.history[static_cast<size_t>(sys) * m.hist_stride + cyc] = e0;
    }
  }
  if (m.drms > 0.0 && rms <= m.drms) {
    if (lane == 0) {
      m.done[sys] = 1;
      line[kLineAct] = 0.0;
    }
    return false;
  }
  // the reference advances its step counter before the gather (hpc_minimization.cu:470)
  const double gam = (cyc + 1 >= m.sd_cycles && gg > 0.0) ? dgg / gg : 0.0;
  double msum = 0.0;
  for (int c = 0; c < natom; c += 32) {
    const int a = c + lane;
    double ms = 0.0;
    if (a < natom) {
      const int gi = base + a;
      const long long ix = d.xfrc[gi];
      const long long iy = d.yfrc[gi];
      const long long iz = d.zfrc[gi];
      if (DBL) {
        double cx = static_cast<double>(ix) * inv_fs;
        double cy = static_cast<double>(iy) * inv_fs;
        double cz = static_cast<double>(iz) * inv_fs;
        if (fabs(gam) > kVeryTiny) {
          cx = fma(gam, m.xcg64[gi], cx);
          cy = fma(gam, m.ycg64[gi], cy);
          cz = fma(gam, m.zcg64[gi], cz);
        }
        m.xcg64[gi] = cx;
        m.ycg64[gi] = cy;
        m.zcg64[gi] = cz;
        ms = cx * cx + cy * cy + cz * cz;
      }
      else {
        float cx = static_cast<float>(static_cast<double>(ix) * inv_fs);
        float cy = static_cast<float>(static_cast<double>(iy) * inv_fs);
        float cz = static_cast<float>(static_cast<double>(iz) * inv_fs);
        if (fabs(gam) > kVeryTiny) {
          const float gf = static_cast<float>(gam);
          cx = fmaf(gf, m.xcg[gi], cx);
          cy = fmaf(gf, m.ycg[gi], cy);
          cz = fmaf(gf, m.zcg[gi], cz);
        }
        m.xcg[gi] = cx;
        m.ycg[gi] = cy;
        m.zcg[gi] = cz;
        ms = static_cast<double>(cx) * cx + static_cast<double>(cy) * cy +
             static_cast<double>(cz) * cz;
      }
      m.xprv[gi] = ix;
      m.yprv[gi] = iy;
      m.zprv[gi] = iz;
    }
    msum += warpSumDouble(ms);
  }
  const double inv_norm = (msum > 0.0) ? 1.0 / sqrt(msum) : 0.0;
  if (lane == 0) {
    line[kLineInvNorm] = inv_norm;
    line[kLineAct] = 1.0;
  }
  return true;
}

// First move of a cycle (line_movement.cui:88-126): record E0 and move along the normalized
// direction by the system's baseline move length
template <bool DBL>
__device__ __forceinline__ void firstMove(const DevSynthesis &d, const DevMinimizer &m, int sys,
                                          double e0, double inv_norm, int lane) {
  const double gpos_scale = 1.0 / d.inv_gpos_scale;
  double* line = m.line + static_cast<size_t>(sys) * kLineFields;
  const double s_move = m.l_move[sys];
  if (lane == 0) {
    line[kLineE0] = e0;
    line[kLineSMove] = s_move;
    line[kLineMfac] = 1.0;
    line[kLineMv1] = 1.0;
  }
  __syncwarp();
  moveSystem<DBL>(d, m, sys, inv_norm * s_move * gpos_scale, lane);
}

// Both at once, the graph minimizer's first line-search kernel of a cycle
template <bool HIST, bool DBL>
__global__ void __launch_bounds__(kLineThreads)
kLineStart(const DevSynthesis d, const DevMinimizer m, int first, int count) {
  const int lane = threadIdx.x & 31;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    const double e0 = systemEnergy(d, sys, lane);
    if (conjugateSystem<HIST, DBL>(d, m, sys, e0, lane)) {
      __syncwarp();
      const double inv_norm = m.line[static_cast<size_t>(sys) * kLineFields + kLineInvNorm];
      firstMove<DBL>(d, m, sys, e0, inv_norm, lane);
    }
  }
}

// The conjugate-gradient step alone (STORMM's launchConjugateGradient)
template <bool HIST, bool DBL>
__global__ void __launch_bounds__(kLineThreads)
kConjugateGradient(const DevSynthesis d, const DevMinimizer m, int first, int count) {
  const int lane = threadIdx.x & 31;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    const double e0 = systemEnergy(d, sys, lane);
    conjugateSystem<HIST, DBL>(d, m, sys, e0, lane);
  }
}

// The first move alone (STORMM's launchLineAdvance with move 0), after kConjugateGradient
template <bool DBL>
__global__ void __launch_bounds__(kLineThreads)
kLineFirstMove(const DevSynthesis d, const DevMinimizer m, int first, int count) {
  const int lane = threadIdx.x & 31;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    const double* line = m.line + static_cast<size_t>(sys) * kLineFields;
    if (line[kLineAct] == 0.0) {
      continue;
    }
    firstMove<DBL>(d, m, sys, systemEnergy(d, sys, lane), line[kLineInvNorm], lane);
  }
}

// Second (move 1) or third (move 2) trial point
template <bool DBL>
__global__ void __launch_bounds__(kLineThreads)
kLineMove(const DevSynthesis d, const DevMinimizer m, int first, int count, int move) {
  const int lane = threadIdx.x & 31;
  const double gpos_scale = 1.0 / d.inv_gpos_scale;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    double* line = m.line + static_cast<size_t>(sys) * kLineFields;
    if (line[kLineAct] == 0.0) {
      continue;
    }
    const double e = systemEnergy(d, sys, lane);
    double mfac;
    if (move == 1) {
      mfac = (e < line[kLineE0]) ? 1.04 : 0.8;
    }
    else {
      mfac = line[kLineMfac] * ((e < line[kLineE1]) ? 1.03 : 0.85);
    }
    const double mv_prev = (move == 1) ? line[kLineMv1] : line[kLineMv2];
    const double step = line[kLineInvNorm] * mfac * line[kLineSMove] * gpos_scale;
    __syncwarp();
    if (lane == 0) {
      line[(move == 1) ? kLineE1 : kLineE2] = e;
      line[kLineMfac] = mfac;
      line[(move == 1) ? kLineMv2 : kLineMv3] = mv_prev + mfac;
    }
    moveSystem<DBL>(d, m, sys, step, lane);
  }
}

// Cubic placement after the third trial point
template <bool DBL>
__global__ void __launch_bounds__(kLineThreads)
kLineFinish(const DevSynthesis d, const DevMinimizer m, int first, int count) {
  const int lane = threadIdx.x & 31;
  const double gpos_scale = 1.0 / d.inv_gpos_scale;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    double* line = m.line + static_cast<size_t>(sys) * kLineFields;
    if (line[kLineAct] == 0.0) {
      continue;
    }
    const double e3 = systemEnergy(d, sys, lane);
    const double ev[4] = {line[kLineE0], line[kLineE1], line[kLineE2], e3};
    const double mv[4] = {0.0, line[kLineMv1], line[kLineMv2], line[kLineMv3]};
    double new_base;
    const double mfac = finalPlacement(ev, mv, &new_base);
    const double s_move = line[kLineSMove];
    const double step = (fabs(mfac) > kVeryTiny) ?
                        line[kLineInvNorm] * mfac * s_move * gpos_scale : 0.0;
    __syncwarp();
    if (lane == 0) {
      m.l_move[sys] = s_move * new_base;
      m.cycle[sys] += 1;
    }
    moveSystem<DBL>(d, m, sys, step, lane);
  }
}

// Final energies after the last cycle into the history
__global__ void __launch_bounds__(kLineThreads)
kLineHistory(const DevSynthesis d, const DevMinimizer m, int first, int count) {
  const int lane = threadIdx.x & 31;
  for (int sys = first + firstWarp(); sys < first + count; sys += warpStride()) {
    const double e = systemEnergy(d, sys, lane);
    const int cyc = m.cycle[sys];
    if (lane == 0 && cyc < m.hist_stride) {
      m.history[static_cast<size_t>(sys) * m.hist_stride + cyc] = e;
    }
  }
}

int lineGrid(int count) {
  const int warps = kLineThreads / 32;
  int b = (count + warps - 1) / warps;
  return b < 1 ? 1 : (b > 4096 ? 4096 : b);
}

}  // namespace

// step: 0 start (conjugate gradient and first move), 1 and 2 trial moves, 3 finish, 4 history
// of the final energies, 5 the conjugate-gradient step alone, 6 the first move alone
cudaError_t launchLineStep(const DevSynthesis &d, const DevMinimizer &m, int first, int count,
                           int step, cudaStream_t stream) {
  if (count <= 0) {
    return cudaSuccess;
  }
  const int grid = lineGrid(count);
  const bool dbl = (m.xcg64 != nullptr);
  switch (step) {
    case 0:
      if (m.history != nullptr) {
        if (dbl) {
          kLineStart<true, true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
        }
        else {
          kLineStart<true, false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
        }
      }
      else if (dbl) {
        kLineStart<false, true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      else {
        kLineStart<false, false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      break;
    case 1:
    case 2:
      if (dbl) {
        kLineMove<true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count, step);
      }
      else {
        kLineMove<false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count, step);
      }
      break;
    case 3:
      if (dbl) {
        kLineFinish<true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      else {
        kLineFinish<false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      break;
    case 4:
      if (m.history != nullptr) {
        kLineHistory<<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      break;
    case 5:
      if (m.history != nullptr) {
        if (dbl) {
          kConjugateGradient<true, true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
        }
        else {
          kConjugateGradient<true, false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
        }
      }
      else if (dbl) {
        kConjugateGradient<false, true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      else {
        kConjugateGradient<false, false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      break;
    case 6:
      if (dbl) {
        kLineFirstMove<true><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      else {
        kLineFirstMove<false><<<grid, kLineThreads, 0, stream>>>(d, m, first, count);
      }
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace sb
