// STORMM's StaticExclusionMask of one topology, built on the host in STORMM's own layout, so a
// caller that keeps STORMM's StaticExclusionMaskSynthesis (Synthesis/static_mask_synthesis.h:54)
// gets bit-identical tables from the same exclusion lists.  The evaluation kernels of this
// library use their own 32 x 32 masks; these tables are for drop-in callers and for checking
// exclusion handling against the reference bit for bit.
//
// Layout (Potential/static_exclusionmask.h:26-41, static_exclusionmask.cpp:20-260):
//   supertiles of 256 atoms; supertile_map_idx[sj * nst + si] is 0 for a supertile without any
//     exclusion, else 256 x (its index among stored supertiles), the offset of its tile map
//   tile_map_idx: 256 entries per stored supertile, entry tj * 16 + ti (16 x 16 atom tiles) is
//     0 for a tile without exclusions, else 32 x (its index among stored tiles)
//   mask_data: 32 words per stored tile (stored tile 0 is all zero): words 0-15 one per i atom
//     with bit j set when the pair is excluded, words 16-31 one per j atom with bit i set
// A tile is stored when it holds an exclusion, lies on the diagonal or is cut short by the end
// of the system; diagonal tiles exclude j >= i, and atoms past the end of the system are
// excluded from everything.  Stored tiles are not deduplicated, as in the reference.
#include <cstdint>
#include <string>
#include <vector>

#include "stormm_b200.h"
#include "synthesis.h"

namespace sb {

namespace {

constexpr int kSuper = 256;                  // atoms per supertile side
constexpr int kTileLen = 16;                 // atoms per tile side
constexpr int kTilesPerSide = kSuper / kTileLen;
constexpr int kTilesPerSuper = kTilesPerSide * kTilesPerSide;

struct StaticMask {
  int nst = 0;
  std::vector<int> super_map;
  std::vector<int> tile_map;
  std::vector<uint32_t> masks;
};

// Does atom i's exclusion list reach any atom in [lo, hi)?
bool reaches(const sb_topology &t, int i, int lo, int hi) {
  for (int k = t.excl_bounds[i]; k < t.excl_bounds[i + 1]; k++) {
    const int j = t.excl_list[k];
    if (j >= lo && j < hi) {
      return true;
    }
  }
  return false;
}

StaticMask build(const sb_topology &t) {
  StaticMask sm;
  const int n = t.natom;
  sm.nst = (n + kSuper - 1) / kSuper;
  sm.super_map.assign(static_cast<size_t>(sm.nst) * sm.nst, 0);
  sm.tile_map.assign(kTilesPerSuper, 0);       // stored supertile 0: the blank map
  sm.masks.assign(2 * kTileLen, 0u);           // stored tile 0: no exclusions
  int stored_super = 1;
  int stored_tiles = 1;
  for (int sti = 0; sti < sm.nst; sti++) {
    const int i0 = sti * kSuper;
    const int i1 = std::min(i0 + kSuper, n);
    for (int stj = 0; stj < sm.nst; stj++) {
      const int j0 = stj * kSuper;
      const int j1 = std::min(j0 + kSuper, n);
      bool any = ((i1 - i0) % kTileLen != 0) || ((j1 - j0) % kTileLen != 0) || (i0 == j0);
      for (int i = i0; i < i1 && !any; i++) {
        any = reaches(t, i, j0, j1);
      }
      if (!any) {
        continue;   // stays 0: the blank supertile
      }
      sm.super_map[static_cast<size_t>(stj) * sm.nst + sti] = stored_super * kTilesPerSuper;
      std::vector<int> map(kTilesPerSuper, 0);
      const int nti = (i1 - i0 + kTileLen - 1) / kTileLen;
      const int ntj = (j1 - j0 + kTileLen - 1) / kTileLen;
      for (int ti = 0; ti < nti; ti++) {
        const int a0 = i0 + ti * kTileLen;
        const int ni = std::min(a0 + kTileLen, i1) - a0;
        for (int tj = 0; tj < ntj; tj++) {
          const int b0 = j0 + tj * kTileLen;
          const int nj = std::min(b0 + kTileLen, j1) - b0;
          uint32_t w[2 * kTileLen] = {};
          bool keep = (ni < kTileLen) || (nj < kTileLen) || (a0 == b0);
          // atoms past the end of the system are excluded from every pair
          uint32_t missing_i = 0u, missing_j = 0u;
          for (int i = ni; i < kTileLen; i++) missing_i |= (1u << i);
          for (int j = nj; j < kTileLen; j++) missing_j |= (1u << j);
          for (int i = ni; i < kTileLen; i++) w[i] = 0xffffffffu;
          for (int j = nj; j < kTileLen; j++) w[kTileLen + j] = 0xffffffffu;
          for (int i = 0; i < kTileLen; i++) w[i] |= missing_j;
          for (int j = 0; j < kTileLen; j++) w[kTileLen + j] |= missing_i;
          if (a0 == b0) {
            // diagonal tile: row i excludes j >= i, column j excludes i <= j
            for (int i = 0; i < kTileLen; i++) {
              w[i] |= 0xffffu & ~((1u << i) - 1u);
              w[kTileLen + i] |= (2u << i) - 1u;
            }
          }
          for (int i = a0; i < a0 + ni; i++) {
            for (int k = t.excl_bounds[i]; k < t.excl_bounds[i + 1]; k++) {
              const int j = t.excl_list[k];
              if (j >= b0 && j < b0 + nj) {
                w[i - a0] |= (1u << (j - b0));
                w[kTileLen + (j - b0)] |= (1u << (i - a0));
                keep = true;
              }
            }
          }
          if (keep) {
            sm.masks.insert(sm.masks.end(), w, w + 2 * kTileLen);
            map[tj * kTilesPerSide + ti] = stored_tiles * 2 * kTileLen;
            stored_tiles++;
          }
        }
      }
      sm.tile_map.insert(sm.tile_map.end(), map.begin(), map.end());
      stored_super++;
    }
  }
  return sm;
}

template <typename T>
void deliver(const std::vector<T> &v, T* out, long long* n, const char* what) {
  if (n == nullptr) {
    throw Error(SB_ERR_ARGUMENT, std::string("null size for ") + what);
  }
  const long long need = static_cast<long long>(v.size());
  if (out != nullptr) {
    if (*n < need) {
      throw Error(SB_ERR_ARGUMENT, std::string("output too small for ") + what);
    }
    std::copy(v.begin(), v.end(), out);
  }
  *n = need;
}

}  // namespace

}  // namespace sb

extern "C" int sb_static_exclusion_mask(const sb_topology* top, int* supertile_stride_count,
                                        int* supertile_map_idx, long long* n_supertile_map,
                                        int* tile_map_idx, long long* n_tile_map,
                                        uint32_t* mask_data, long long* n_mask_data) {
  try {
    if (top == nullptr || top->natom <= 0 || top->excl_bounds == nullptr ||
        (top->excl_list == nullptr && top->excl_bounds[top->natom] > 0)) {
      throw sb::Error(SB_ERR_ARGUMENT, "a topology with atoms and exclusion lists is required");
    }
    const sb::StaticMask sm = sb::build(*top);
    if (supertile_stride_count != nullptr) {
      *supertile_stride_count = sm.nst;
    }
    sb::deliver(sm.super_map, supertile_map_idx, n_supertile_map, "the supertile map");
    sb::deliver(sm.tile_map, tile_map_idx, n_tile_map, "the tile map");
    sb::deliver(sm.masks, mask_data, n_mask_data, "the mask data");
    return SB_OK;
  }
  catch (const sb::Error &e) {
    sb::setLastError(e.what());
    return e.code;
  }
  catch (const std::exception &e) {
    sb::setLastError(e.what());
    return SB_ERR_ARGUMENT;
  }
}
