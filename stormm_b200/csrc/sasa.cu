// Solvent-accessible surface area by sphere points, as STORMM's MM-GBSA application scores it
// (Potential/surface_area.tpp:28-161 with the Lennard-Jones radii of surface_area.tpp:163-173).
//
// One block per system, in FP64 throughout.  Each atom carries a sphere of points at its radius
// plus the probe; a point survives unless it lies strictly inside another atom's probe-enlarged
// sphere.  The reference bins atoms into cells of at least twice the largest probe-enlarged
// radius over the system's bounding box and tests a point of an atom in cell (i, j, k) only
// against atoms in cells i-1..i, j-1..j, k-1..k (its loop bounds stop below the upper
// neighbours); the kernel applies the same cell rule, so the surviving points are the same.
// A system with no extent along an axis has no cells there and scores zero, as in the reference.
// Point, displacement and distance arithmetic use round-to-nearest multiplies and adds without
// fused multiply-add, in the reference's order, so each point's verdict is the host's.
#include <cuda_runtime.h>

#include "device_kits.h"

namespace sb {
namespace {

constexpr int kSasaThreads = 256;

__device__ __forceinline__ double blockReduce(double v, bool take_max, double* scratch) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = take_max ? fmax(v, w) : fmin(v, w);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (kSasaThreads >> 5)) ? scratch[lane] : scratch[0];
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = take_max ? fmax(v, w) : fmin(v, w);
    }
    if (lane == 0) scratch[0] = v;
  }
  __syncthreads();
  const double out = scratch[0];
  __syncthreads();
  return out;
}

__device__ __forceinline__ int cellOf(double x, double origin, double width, int count) {
  int c = static_cast<int>(__ddiv_rn(__dsub_rn(x, origin), width));
  return c < 0 ? 0 : (c >= count ? count - 1 : c);
}

// cell: per-atom scratch (padded layout) for the packed cell coordinates
__global__ void __launch_bounds__(kSasaThreads)
kSurfaceArea(const long long* xcrd, const long long* ycrd, const long long* zcrd,
             double inv_gpos_scale, const int* atom_start, const int* atom_count,
             const double* radius, const double3* pts, int npts, double probe, double weight,
             int* cell, double* out) {
  __shared__ double scratch[32];
  const int sys = blockIdx.x;
  const int base = atom_start[sys], n = atom_count[sys];
  double lo[3] = {1.0e300, 1.0e300, 1.0e300}, hi[3] = {-1.0e300, -1.0e300, -1.0e300};
  double rmax = 0.0;
  for (int i = threadIdx.x; i < n; i += kSasaThreads) {
    const double x[3] = {static_cast<double>(xcrd[base + i]) * inv_gpos_scale,
                         static_cast<double>(ycrd[base + i]) * inv_gpos_scale,
                         static_cast<double>(zcrd[base + i]) * inv_gpos_scale};
    for (int d = 0; d < 3; d++) {
      lo[d] = fmin(lo[d], x[d]);
      hi[d] = fmax(hi[d], x[d]);
    }
    rmax = fmax(rmax, radius[base + i]);
  }
  double origin[3], len[3];
  for (int d = 0; d < 3; d++) {
    origin[d] = blockReduce(lo[d], false, scratch);
    len[d] = __dsub_rn(blockReduce(hi[d], true, scratch), origin[d]);
  }
  rmax = blockReduce(rmax, true, scratch);
  const double min_width = 2.0 * __dadd_rn(rmax, probe);
  int count[3];
  double width[3];
  for (int d = 0; d < 3; d++) {
    count[d] = static_cast<int>(ceil(__ddiv_rn(len[d], min_width)));
    width[d] = __ddiv_rn(len[d], static_cast<double>(count[d]));
  }
  if (count[0] == 0 || count[1] == 0 || count[2] == 0) {
    if (threadIdx.x == 0) out[sys] = 0.0;
    return;
  }
  if (count[0] > 1024 || count[1] > 1024 || count[2] > 1024) {
    // more cells along an axis than the packed cell index holds (an extent of kilometres)
    if (threadIdx.x == 0) out[sys] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  for (int i = threadIdx.x; i < n; i += kSasaThreads) {
    const int cx = cellOf(static_cast<double>(xcrd[base + i]) * inv_gpos_scale, origin[0],
                          width[0], count[0]);
    const int cy = cellOf(static_cast<double>(ycrd[base + i]) * inv_gpos_scale, origin[1],
                          width[1], count[1]);
    const int cz = cellOf(static_cast<double>(zcrd[base + i]) * inv_gpos_scale, origin[2],
                          width[2], count[2]);
    cell[base + i] = (cz << 20) | (cy << 10) | cx;
  }
  __syncthreads();
  // area per surviving point of atom m: (4 pi / npts) r^2
  const double patch = __ddiv_rn(4.0 * 3.141592653589793, static_cast<double>(npts));
  double area = 0.0;
  const long long work = static_cast<long long>(n) * npts;
  for (long long w = threadIdx.x; w < work; w += kSasaThreads) {
    const int m = static_cast<int>(w / npts), p = static_cast<int>(w % npts);
    const double ax = static_cast<double>(xcrd[base + m]) * inv_gpos_scale;
    const double ay = static_cast<double>(ycrd[base + m]) * inv_gpos_scale;
    const double az = static_cast<double>(zcrd[base + m]) * inv_gpos_scale;
    const double r_eff = __dadd_rn(radius[base + m], probe);
    const double3 s = pts[p];
    const double px = __dadd_rn(ax, __dmul_rn(s.x, r_eff));
    const double py = __dadd_rn(ay, __dmul_rn(s.y, r_eff));
    const double pz = __dadd_rn(az, __dmul_rn(s.z, r_eff));
    const int cm = cell[base + m];
    const int mx = cm & 1023, my = (cm >> 10) & 1023, mz = cm >> 20;
    bool survives = true;
    for (int v = 0; v < n && survives; v++) {
      if (v == m) continue;
      const int cv = cell[base + v];
      const int vx = cv & 1023, vy = (cv >> 10) & 1023, vz = cv >> 20;
      if (vx > mx || vx < mx - 1 || vy > my || vy < my - 1 || vz > mz || vz < mz - 1) continue;
      const double dx = __dsub_rn(px, static_cast<double>(xcrd[base + v]) * inv_gpos_scale);
      const double dy = __dsub_rn(py, static_cast<double>(ycrd[base + v]) * inv_gpos_scale);
      const double dz = __dsub_rn(pz, static_cast<double>(zcrd[base + v]) * inv_gpos_scale);
      const double rv = __dadd_rn(radius[base + v], probe);
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                  __dmul_rn(dz, dz));
      if (d2 < __dmul_rn(rv, rv)) survives = false;
    }
    if (survives) area += __dmul_rn(__dmul_rn(patch, r_eff), r_eff);
  }
  // a block sum of the per-thread areas
  for (int o = 16; o > 0; o >>= 1) area += __shfl_xor_sync(0xffffffffu, area, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) scratch[warp] = area;
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int k = 0; k < (kSasaThreads >> 5); k++) total += scratch[k];
    out[sys] = total * weight;
  }
}

}  // namespace

cudaError_t launchSurfaceArea(const long long* xcrd, const long long* ycrd,
                              const long long* zcrd, double inv_gpos_scale,
                              const int* atom_start, const int* atom_count, int nsys,
                              const double* radius, const double3* pts, int npts, double probe,
                              double weight, int* cell, double* out, cudaStream_t stream) {
  if (nsys <= 0) return cudaSuccess;
  kSurfaceArea<<<nsys, kSasaThreads, 0, stream>>>(xcrd, ycrd, zcrd, inv_gpos_scale, atom_start,
                                                  atom_count, radius, pts, npts, probe, weight,
                                                  cell, out);
  return cudaGetLastError();
}

}  // namespace sb
