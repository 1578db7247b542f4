// Line-search arithmetic shared by the persistent minimizer (minimize.cu) and the graph
// minimizer's per-system kernels (line_search.cu): the reference's move factors and the cubic
// placement of MolecularMechanics/line_movement.cui:88-336, in FP64.
#ifndef STORMM_B200_LINE_SEARCH_CUH
#define STORMM_B200_LINE_SEARCH_CUH

#include <cuda_runtime.h>

namespace sb {

namespace {

constexpr double kVeryTiny = 1.0e-12;   // Constants/scaling.h verytiny

__device__ __forceinline__ double warpSumDouble(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// Cubic through (0, e0), (x1, e1), (x2, e2), (x3, e3): Gauss-Jordan elimination with partial
// pivoting on the 4 x 4 Vandermonde system, the elimination line_movement.cui:160-236 performs
__device__ void cubicFit(const double* x, const double* e, double* abcd) {
  double mtx[4][5];
  for (int r = 0; r < 4; r++) {
    mtx[r][0] = x[r] * x[r] * x[r];
    mtx[r][1] = x[r] * x[r];
    mtx[r][2] = x[r];
    mtx[r][3] = 1.0;
    mtx[r][4] = e[r];
  }
  for (int col = 0; col < 4; col++) {
    int piv = col;
    for (int r = col + 1; r < 4; r++) {
      if (fabs(mtx[r][col]) > fabs(mtx[piv][col])) piv = r;
    }
    if (piv != col) {
      for (int q = 0; q < 5; q++) {
        const double t = mtx[col][q];
        mtx[col][q] = mtx[piv][q];
        mtx[piv][q] = t;
      }
    }
    const double p = mtx[col][col];
    for (int q = 0; q < 5; q++) mtx[col][q] /= p;
    for (int r = 0; r < 4; r++) {
      if (r == col) continue;
      const double f = mtx[r][col];
      for (int q = 0; q < 5; q++) mtx[r][q] -= f * mtx[col][q];
    }
  }
  for (int r = 0; r < 4; r++) abcd[r] = mtx[r][4];
}

// Final placement along the line from the four energies (line_movement.cui:236-336): returns the
// move factor relative to the third trial point and sets the next move length's scale
__device__ double finalPlacement(const double* ev, const double* mv, double* new_base) {
  if (ev[0] < ev[1] && ev[0] < ev[2] && ev[0] < ev[3]) {
    *new_base = 0.8;
    return -mv[3];
  }
  double abcd[4];
  cubicFit(mv, ev, abcd);
  const double d0 = 3.0 * abcd[0], d1 = 2.0 * abcd[1], d2 = abcd[2];
  const double sqrt_arg = d1 * d1 - 4.0 * d0 * d2;
  if (sqrt_arg < 0.0) {
    if (ev[0] < ev[3]) {
      *new_base = 0.8;
      return -mv[3];
    }
    *new_base = 1.2;
    return 0.0;
  }
  const double ext_i = (-d1 + sqrt(sqrt_arg)) / (2.0 * d0);
  const double ext_ii = (-d1 - sqrt(sqrt_arg)) / (2.0 * d0);
  const double min_pos = (2.0 * d0 * ext_i + d1 > 0.0) ? ext_i : ext_ii;
  if (min_pos <= 0.0) {
    if (ev[3] >= ev[0]) {
      *new_base = 0.8;
      return -mv[3];
    }
    *new_base = 1.2;
    return 0.0;
  }
  if (min_pos < mv[3]) {
    const double epred = ((abcd[0] * min_pos + abcd[1]) * min_pos + abcd[2]) * min_pos + abcd[3];
    if (epred > ev[0]) {
      *new_base = 0.8;
      return -mv[3];
    }
    if (epred < ev[3]) {
      *new_base = (min_pos > 0.6) ? 1.05 : 0.95;
      return min_pos - mv[3];
    }
    *new_base = 1.05;
    return 0.0;
  }
  *new_base = 1.05;
  return 0.0;
}

}  // namespace

}  // namespace sb

#endif
