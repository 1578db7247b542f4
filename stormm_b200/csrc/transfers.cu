// Conversions between the caller's unpadded double-precision arrays and the synthesis'
// fixed-point device layout, done on the device so that a host round trip is one copy each way.
//
//   coordinates  double (A) -> int64 with gpos_bits fraction bits, overflow word cleared
//                (STORMM's PhaseSpaceSynthesis import, Synthesis/phasespace_synthesis.cpp)
//   forces       int95 (int64 + int32 overflow) -> double (kcal/mol/A)
//   energies     int64 per system and slot -> double (kcal/mol)
#include <cuda_runtime.h>

#include "device_kits.h"
#include "fixed_point.cuh"

namespace sb {

namespace {

// One thread per atom: map[a] is the padded index of unpadded atom a
__global__ void kImportCoordinates(const double* __restrict__ xyz, const int* __restrict__ map,
                                   int natom, double scale, long long* xcrd, long long* ycrd,
                                   long long* zcrd, int* xo, int* yo, int* zo, int* status) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < natom; a += gridDim.x * blockDim.x) {
    const int gi = map[a];
    const double x = xyz[3 * a] * scale;
    const double y = xyz[3 * a + 1] * scale;
    const double z = xyz[3 * a + 2] * scale;
    const double lim = 9.0e18;
    if (!(fabs(x) < lim && fabs(y) < lim && fabs(z) < lim)) {
      // not finite or beyond the int64 range: flag it, leave the atom where it was
      atomicOr(status, 2);
      continue;
    }
    xcrd[gi] = __double2ll_rn(x);
    ycrd[gi] = __double2ll_rn(y);
    zcrd[gi] = __double2ll_rn(z);
    xo[gi] = 0;
    yo[gi] = 0;
    zo[gi] = 0;
  }
}

__global__ void kExportCoordinates(const long long* __restrict__ xcrd,
                                   const long long* __restrict__ ycrd,
                                   const long long* __restrict__ zcrd,
                                   const int* __restrict__ map, int natom, double inv_scale,
                                   double* xyz) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < natom; a += gridDim.x * blockDim.x) {
    const int gi = map[a];
    xyz[3 * a] = static_cast<double>(xcrd[gi]) * inv_scale;
    xyz[3 * a + 1] = static_cast<double>(ycrd[gi]) * inv_scale;
    xyz[3 * a + 2] = static_cast<double>(zcrd[gi]) * inv_scale;
  }
}

__global__ void kExportForces(const long long* __restrict__ xf, const long long* __restrict__ yf,
                              const long long* __restrict__ zf, const int* __restrict__ xo,
                              const int* __restrict__ yo, const int* __restrict__ zo,
                              const int* __restrict__ map, int natom, double inv_scale,
                              double* xyz) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < natom; a += gridDim.x * blockDim.x) {
    const int gi = map[a];
    xyz[3 * a] = int95ToDouble(xf[gi], xo[gi]) * inv_scale;
    xyz[3 * a + 1] = int95ToDouble(yf[gi], yo[gi]) * inv_scale;
    xyz[3 * a + 2] = int95ToDouble(zf[gi], zo[gi]) * inv_scale;
  }
}

__global__ void kExportEnergies(const unsigned long long* __restrict__ nrg, int n,
                                double inv_scale, double* out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    out[e] = static_cast<double>(static_cast<long long>(nrg[e])) * inv_scale;
  }
}

// Zero several arrays in one launch: each block walks every array in 16-byte words
__global__ void kClear(ClearList list) {
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int a = 0; a < list.count; a++) {
    uint4* p = reinterpret_cast<uint4*>(list.ptr[a]);
    const size_t n = list.words[a];
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += stride) {
      p[i] = zero;
    }
  }
}

int gridFor(int n) {
  const int b = (n + 255) / 256;
  return b < 1 ? 1 : (b > 4096 ? 4096 : b);
}

}  // namespace

cudaError_t launchImportCoordinates(const double* d_xyz, const int* d_map, int natom,
                                    double scale, long long* xcrd, long long* ycrd,
                                    long long* zcrd, int* xo, int* yo, int* zo, int* status,
                                    cudaStream_t stream) {
  kImportCoordinates<<<gridFor(natom), 256, 0, stream>>>(d_xyz, d_map, natom, scale, xcrd, ycrd,
                                                         zcrd, xo, yo, zo, status);
  return cudaGetLastError();
}

cudaError_t launchExportCoordinates(const long long* xcrd, const long long* ycrd,
                                    const long long* zcrd, const int* d_map, int natom,
                                    double inv_scale, double* d_xyz, cudaStream_t stream) {
  kExportCoordinates<<<gridFor(natom), 256, 0, stream>>>(xcrd, ycrd, zcrd, d_map, natom,
                                                         inv_scale, d_xyz);
  return cudaGetLastError();
}

cudaError_t launchExportForces(const long long* xf, const long long* yf, const long long* zf,
                               const int* xo, const int* yo, const int* zo, const int* d_map,
                               int natom, double inv_scale, double* d_xyz, cudaStream_t stream) {
  kExportForces<<<gridFor(natom), 256, 0, stream>>>(xf, yf, zf, xo, yo, zo, d_map, natom,
                                                    inv_scale, d_xyz);
  return cudaGetLastError();
}

cudaError_t launchClear(const ClearList &list, int sm_count, cudaStream_t stream) {
  size_t most = 0;
  for (int a = 0; a < list.count; a++) {
    if (reinterpret_cast<uintptr_t>(list.ptr[a]) % 16 != 0) return cudaErrorInvalidValue;
    most = (list.words[a] > most) ? list.words[a] : most;
  }
  if (list.count == 0 || most == 0) return cudaSuccess;
  size_t blocks = (most + 255) / 256;
  const size_t cap = static_cast<size_t>(sm_count > 0 ? sm_count : 148) * 8;
  blocks = (blocks > cap) ? cap : blocks;
  kClear<<<static_cast<int>(blocks), 256, 0, stream>>>(list);
  return cudaGetLastError();
}

cudaError_t launchExportEnergies(const unsigned long long* nrg, int n, double inv_scale,
                                 double* d_out, cudaStream_t stream) {
  kExportEnergies<<<gridFor(n), 256, 0, stream>>>(nrg, n, inv_scale, d_out);
  return cudaGetLastError();
}

}  // namespace sb
