// Split fixed-point accumulation in STORMM's formats.
//
// int63: value = overflow * 2^31 + primary, with an int32 primary and an int32 overflow word.
// int95: value = overflow * 2^63 + primary, with an int64 primary and an int32 overflow word.
// (Numerics/split_fixed_precision.h:30-34, Numerics/accumulation.cui:18-206.)  Additions are
// integer and therefore independent of order, which makes every sum bit-identical from run to
// run.  A primary that wraps when a contribution is added is detected from the sign pattern and
// the overflow word takes the carry of +/-2 (one wrap of the primary is 2^32 = 2 * 2^31 units).
#ifndef STORMM_B200_FIXED_POINT_CUH
#define STORMM_B200_FIXED_POINT_CUH

namespace sb {

constexpr float kInt63Unit = 2147483648.0f;              // 2^31
constexpr double kInt95Unit = 9223372036854775808.0;     // 2^63

// Real value (already scaled) -> int63 pair (primary, overflow)
__device__ __forceinline__ int2 toInt63(float v) {
  int2 r;
  if (fabsf(v) >= kInt63Unit) {
    const int spill = static_cast<int>(v / kInt63Unit);
    r.x = __float2int_rn(v - static_cast<float>(spill) * kInt63Unit);
    r.y = spill;
  }
  else {
    r.x = __float2int_rn(v);
    r.y = 0;
  }
  return r;
}

// Add a scaled real value to an int63 accumulator held as two int arrays (shared or global)
__device__ __forceinline__ void atomicAddInt63(float v, int* primary, int* overflow) {
  const int2 iv = toInt63(v);
  const int old = atomicAdd(primary, iv.x);
  const int sum = old + iv.x;
  int carry = iv.y;
  if (((old ^ sum) < 0) && ((old ^ iv.x) >= 0)) {
    carry += (iv.x < 0) ? -2 : 2;
  }
  if (carry != 0) {
    atomicAdd(overflow, carry);
  }
}

// A fixed-point coordinate (already scaled to Angstroms) as an FP32 pair hi + lo with hi on a
// 2^-10 A grid.  For |x| < 8192 A and a coordinate grid of up to 2^-35 A, hi + lo == x exactly,
// and for two atoms both hi_j - hi_i and lo_j - lo_i are exact in FP32 (hi differences are below
// 2^24 units of 2^-10, lo differences below 2^22 units of 2^-32), so their sum rounds the exact
// separation once and that rounding's error is lo_d - (d - hi_d), recoverable in two additions
// (separationError).  An unconstrained hi = (float)x loses both properties.
__device__ __forceinline__ void splitCoordinate(double x, float* hi, float* lo) {
  const double h = rint(x * 1024.0) * 0.0009765625;
  *hi = static_cast<float>(h);
  *lo = static_cast<float>(x - h);
}

// Rounding error of d = hd + ld, where hd and ld are separations of hi and lo parts from
// splitCoordinate: the exact separation is d + separationError(hd, ld, d)
__device__ __forceinline__ float separationError(float hd, float ld, float d) {
  return __fsub_rn(ld, __fsub_rn(d, hd));
}

// int63 pair -> int64
__device__ __forceinline__ long long int63ToLong(int primary, int overflow) {
  return static_cast<long long>(overflow) * 2147483648LL + static_cast<long long>(primary);
}

// Add an int64 to an int95 accumulator (primary int64, overflow int32) held in global memory by
// one owner (no concurrent writers): read-modify-write with carry detection.
__device__ __forceinline__ void addInt95(long long v, long long* primary, int* overflow) {
  const long long old = *primary;
  const long long sum = static_cast<long long>(static_cast<unsigned long long>(old) +
                                               static_cast<unsigned long long>(v));
  *primary = sum;
  if (((old ^ sum) < 0) && ((old ^ v) >= 0)) {
    *overflow += (v < 0) ? -2 : 2;
  }
}

// int95 pair -> double
__device__ __forceinline__ double int95ToDouble(long long primary, int overflow) {
  return static_cast<double>(overflow) * kInt95Unit + static_cast<double>(primary);
}

// double -> int95 pair
__device__ __forceinline__ void toInt95(double v, long long* primary, int* overflow) {
  if (fabs(v) >= kInt95Unit) {
    const int spill = static_cast<int>(v / kInt95Unit);
    *primary = __double2ll_rn(v - static_cast<double>(spill) * kInt95Unit);
    *overflow = spill;
  }
  else {
    *primary = __double2ll_rn(v);
    *overflow = 0;
  }
}

}  // namespace sb

#endif
