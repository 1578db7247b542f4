// Tile tasks of the molecules on the tiled path (DevTiled): every 32 x 32 tile of every such
// molecule is an independent warp task, found from a global tile index by binary search over
// the molecules' tile prefix.  Shared by the FP32 tile kernels (tiled.cu) and the FP64 mode
// (fp64.cu).
#ifndef STORMM_B200_TILE_TASKS_CUH
#define STORMM_B200_TILE_TASKS_CUH

#include <cuda_runtime.h>

#include "unit_eval.cuh"

namespace sb {

namespace {

constexpr int kTiledWarps = 8;            // warps per block of the tile kernels

// Tiled molecule and tile within it of global tile index g
__device__ __forceinline__ int tiledOwner(const DevTiled &t, int g) {
  int lo = 0, hi = t.nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.tile_prefix[mid] <= g) {
      lo = mid;
    }
    else {
      hi = mid - 1;
    }
  }
  return lo;
}

__device__ __forceinline__ TileInfo tiledTileInfo(const DevSynthesis &d, int sysid, int local,
                                                  int* I, int* J) {
  tileCoordinates(local, I, J);
  const int n = d.atom_count[sysid];
  TileInfo ti;
  ti.k = 0;
  ti.local = local;
  ti.diag = (*I == *J);
  ti.ibase = 0;
  ti.jbase = ti.diag ? 0 : kTile;
  ti.ni = min(kTile, n - *I * kTile);
  ti.nj = min(kTile, n - *J * kTile);
  return ti;
}

// The warp's contiguous run of tiles [first, last)
__device__ __forceinline__ void warpTileRange(const DevTiled &t, int tile_begin, int tile_end,
                                              int* first, int* last) {
  const int nwarps = gridDim.x * kTiledWarps;
  const int w = blockIdx.x * kTiledWarps + (threadIdx.x >> 5);
  const int n = tile_end - tile_begin;
  const int per = (n + nwarps - 1) / nwarps;
  *first = tile_begin + min(n, w * per);
  *last = tile_begin + min(n, (w + 1) * per);
}

// Tiled molecule owning padded position q of the tiled atoms, and the atom's global index
__device__ __forceinline__ int tiledAtom(const DevSynthesis &d, const DevTiled &t, int q,
                                         int* sysid, int* a) {
  int lo = 0, hi = t.nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.atom_prefix[mid] <= q) {
      lo = mid;
    }
    else {
      hi = mid - 1;
    }
  }
  *sysid = t.systems[lo];
  *a = q - t.atom_prefix[lo];
  return d.atom_start[*sysid] + *a;
}

inline int tileGrid(int ntiles, int sm_count) {
  const int want = (ntiles + kTiledWarps * 4 - 1) / (kTiledWarps * 4);   // about 4 tiles a warp
  const int cap = sm_count * 8;
  return want < 1 ? 1 : (want > cap ? cap : want);
}

inline int atomGrid(int natom, int sm_count) {
  const int want = (natom + 255) / 256;
  const int cap = sm_count * 8;
  return want < 1 ? 1 : (want > cap ? cap : want);
}

}  // namespace

}  // namespace sb

#endif
