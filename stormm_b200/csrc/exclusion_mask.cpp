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
#include <algorithm>
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

// ------------------------------------------------------------------------------------------------
// Synthesis of many systems (Synthesis/static_mask_synthesis.cpp:84-200): the per-topology
// tables concatenated, the blank supertile and blank tile shared, every stored index shifted by
// what earlier topologies stored; systems sharing a topology share its tables.
// ------------------------------------------------------------------------------------------------
struct MaskSynthesis {
  std::vector<int> atom_counts, atom_offsets, super_bounds, super_map, tile_map;
  std::vector<uint32_t> masks;
};

void checkSynthesisArgs(const sb_topology* tops, int ntop, const int* topology_index, int nsys) {
  if (tops == nullptr || ntop <= 0 || topology_index == nullptr || nsys <= 0) {
    throw Error(SB_ERR_ARGUMENT, "topologies and systems are required");
  }
  for (int t = 0; t < ntop; t++) {
    if (tops[t].natom <= 0 || tops[t].excl_bounds == nullptr ||
        (tops[t].excl_list == nullptr && tops[t].excl_bounds[tops[t].natom] > 0)) {
      throw Error(SB_ERR_ARGUMENT, "topology " + std::to_string(t) +
                  " needs atoms and exclusion lists");
    }
  }
  for (int s = 0; s < nsys; s++) {
    if (topology_index[s] < 0 || topology_index[s] >= ntop) {
      throw Error(SB_ERR_ARGUMENT, "topology index of system " + std::to_string(s) +
                  " out of range");
    }
  }
}

MaskSynthesis buildSynthesis(const sb_topology* tops, int ntop, const int* topology_index,
                             int nsys) {
  std::vector<StaticMask> base(static_cast<size_t>(ntop));
  std::vector<int> super_shift(ntop), tile_shift(ntop);
  int n_super = 1, n_tiles = 1;
  for (int t = 0; t < ntop; t++) {
    base[t] = build(tops[t]);
    super_shift[t] = n_super * kTilesPerSuper;
    tile_shift[t] = n_tiles * 2 * kTileLen;
    n_super += static_cast<int>(base[t].tile_map.size()) / kTilesPerSuper - 1;
    n_tiles += static_cast<int>(base[t].masks.size()) / (2 * kTileLen) - 1;
  }
  MaskSynthesis ms;
  ms.super_bounds.push_back(0);
  int offset = 0;
  for (int s = 0; s < nsys; s++) {
    const int t = topology_index[s];
    const StaticMask &b = base[t];
    ms.atom_counts.push_back(tops[t].natom);
    ms.atom_offsets.push_back(offset);
    offset += ((tops[t].natom + 31) / 32) * 32;
    for (int v : b.super_map) {
      ms.super_map.push_back(v == 0 ? 0 : v + super_shift[t] - kTilesPerSuper);
    }
    ms.super_bounds.push_back(static_cast<int>(ms.super_map.size()));
  }
  ms.tile_map.assign(kTilesPerSuper, 0);
  ms.masks.assign(2 * kTileLen, 0u);
  for (int t = 0; t < ntop; t++) {
    const StaticMask &b = base[t];
    ms.masks.insert(ms.masks.end(), b.masks.begin() + 2 * kTileLen, b.masks.end());
    for (size_t i = kTilesPerSuper; i < b.tile_map.size(); i++) {
      const int v = b.tile_map[i];
      ms.tile_map.push_back(v == 0 ? 0 : v + tile_shift[t] - 2 * kTileLen);
    }
  }
  return ms;
}

// ------------------------------------------------------------------------------------------------
// STORMM's nonbonded work units of the TILE_GROUPS kind (Synthesis/nonbonded_workunit.cpp:454-755,
// nonbonded_workunit.tpp:8-150, AtomGraphSynthesis::loadNonbondedWorkUnits in
// ag_synthesis_mechanics.cpp:2668-2730).  Tiles are 16 x 16 atoms; a work unit imports at most 20
// tile edges (320 atoms) and aims for 8, 16, 32 or 64 tiles, the smallest target that keeps the
// work-unit count under 2K, 4K, 8K or 128K.
// ------------------------------------------------------------------------------------------------
constexpr int kMaxImports = 320 / kTileLen;        // 20
constexpr int kTileBatch = 8;                      // tiles per warp batch
constexpr int kAbstractLength = 64;
constexpr int kRefreshBlock = 256;

struct Tile {
  int x, y, sys;
};

struct WorkUnit {
  std::vector<Tile> tiles;
  int import_count = 0;
  std::vector<int> imports, import_sys, size_keys;
  std::vector<uint32_t> insr_x, insr_y;
  int init_mask = 0, refresh_start = 0, refresh_code = 0;
};

// A work unit from its tile list: unique imports in (system, tile) order, tile instructions
// naming the two imports (16 x import slot, the ordinate's shifted 16 bits) and the tile's mask
// in the synthesis tables, and the packed import sizes
WorkUnit makeWorkUnit(const MaskSynthesis &ms, const std::vector<Tile> &tiles) {
  WorkUnit wu;
  wu.tiles = tiles;
  const int nt = static_cast<int>(tiles.size());
  wu.insr_x.assign(nt, 0u);
  wu.insr_y.assign(nt, 0u);
  std::vector<long long> keys;
  for (int i = 0; i < nt; i++) {
    const Tile &t = tiles[i];
    const int natom = ms.atom_counts[t.sys];
    const int nst = (natom + kSuper - 1) / kSuper;
    const int sti = t.x / kTilesPerSide, stj = t.y / kTilesPerSide;
    const int st_entry = ms.super_map[ms.super_bounds[t.sys] + stj * nst + sti];
    const int ti = t.x - sti * kTilesPerSide, tj = t.y - stj * kTilesPerSide;
    wu.insr_y[i] = static_cast<uint32_t>(ms.tile_map[st_entry + tj * kTilesPerSide + ti]);
    keys.push_back((static_cast<long long>(t.sys) << 32) | t.x);
    keys.push_back((static_cast<long long>(t.sys) << 32) | t.y);
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  wu.import_count = static_cast<int>(keys.size());
  wu.imports.assign(kMaxImports, -1);
  wu.import_sys.assign(kMaxImports, 0);
  wu.size_keys.assign(kMaxImports / 4, 0);
  for (int i = 0; i < wu.import_count && i < kMaxImports; i++) {
    const int sys = static_cast<int>(keys[i] >> 32);
    const int tile = static_cast<int>(keys[i] & 0xffffffffLL);
    wu.import_sys[i] = sys;
    wu.imports[i] = tile * kTileLen + ms.atom_offsets[sys];
    for (int k = 0; k < nt; k++) {
      if (tiles[k].sys == sys && tiles[k].x == tile) {
        wu.insr_x[k] |= static_cast<uint32_t>(kTileLen * i);
      }
      if (tiles[k].sys == sys && tiles[k].y == tile) {
        wu.insr_x[k] |= static_cast<uint32_t>(kTileLen * i) << 16;
      }
    }
    const int limit = ms.atom_offsets[sys] + ms.atom_counts[sys];
    const int batch = std::min(limit - wu.imports[i], kTileLen);
    wu.size_keys[i / 4] |= batch << (8 * (i % 4));
  }
  return wu;
}

// Imports a tile would add to the unit, given which tile edges it already holds
int newImports(const std::vector<char> &held, int base, const Tile &t) {
  return (t.x == t.y) ? 1 - held[base + t.x] : 2 - held[base + t.x] - held[base + t.y];
}

std::vector<WorkUnit> enumerateWorkUnits(const MaskSynthesis &ms, int target) {
  const int nsys = static_cast<int>(ms.atom_counts.size());
  std::vector<int> edge_start(nsys);
  int edges = 0;
  for (int s = 0; s < nsys; s++) {
    edge_start[s] = edges;
    edges += (ms.atom_counts[s] + kTileLen - 1) / kTileLen;
  }
  std::vector<char> held(edges, 0);
  std::vector<Tile> cur;
  int imports = 0;
  std::vector<WorkUnit> out;
  auto add = [&](const Tile &t) -> bool {
    const int base = edge_start[t.sys];
    const int grow = newImports(held, base, t);
    if (imports + grow > kMaxImports) {
      return false;
    }
    imports += grow;
    held[base + t.x] = 1;
    held[base + t.y] = 1;
    cur.push_back(t);
    return true;
  };
  auto release = [&]() {
    for (const Tile &t : cur) {
      held[edge_start[t.sys] + t.x] = 0;
      held[edge_start[t.sys] + t.y] = 0;
    }
    cur.clear();
    imports = 0;
  };
  // Ordinate bands two, four, six or eight tile edges wide; the abscissa sweeps up and down
  // alternately, tiles on or below the diagonal only
  const int band = (target == 8) ? 2 : (target == 16) ? 4 : (target == 32) ? 6 : 8;
  for (int s = 0; s < nsys; s++) {
    const int n_edge = (ms.atom_counts[s] + kTileLen - 1) / kTileLen;
    int lo = 0;
    int hi = std::min(band, n_edge);
    bool upward = true;
    while (lo < n_edge) {
      for (int step = 0; step < n_edge; step++) {
        const int i = upward ? step : n_edge - 1 - step;
        for (int j = lo; j < hi; j++) {
          if (j > i) {
            continue;
          }
          const Tile t = {i, j, s};
          if (add(t)) {
            if (static_cast<int>(cur.size()) == target) {
              out.push_back(makeWorkUnit(ms, cur));
              release();
            }
            continue;
          }
          // The import limit is reached: commit the largest multiple of eight tiles, carry the
          // rest and this tile into the next unit
          const int keep = (static_cast<int>(cur.size()) / kTileBatch) * kTileBatch;
          const std::vector<Tile> carry(cur.begin() + keep, cur.end());
          out.push_back(makeWorkUnit(ms, std::vector<Tile>(cur.begin(), cur.begin() + keep)));
          release();
          for (const Tile &c : carry) {
            add(c);
          }
          add(t);
        }
      }
      upward = !upward;
      lo = hi;
      hi = std::min(lo + band, n_edge);
    }
  }
  out.push_back(makeWorkUnit(ms, cur));      // the last unit, even when it is empty
  release();

  // Initialization masks: bit j when this unit is the first to import its jth tile edge
  std::vector<char> first_seen(static_cast<size_t>(ms.atom_offsets.back()) +
                               ((ms.atom_counts.back() + 31) / 32) * 32 + 1, 0);
  for (WorkUnit &wu : out) {
    int mask = 0;
    for (int j = 0; j < wu.import_count; j++) {
      const int a = wu.imports[j];
      if (!first_seen[a]) {
        first_seen[a] = 1;
        mask |= (1 << j);
      }
    }
    wu.init_mask = mask;
  }
  return out;
}

// Accumulator refresh assignments (nonbonded_workunit.cpp:573-700): which atoms each unit
// clears for the next cycle, by STORMM's InitializationTask, without a GPU in view (no units
// are added for random-number work)
int initializationCode(int task, int cache_depth) {
  switch (task) {
  case 0: return 7;                              // GENERAL_DYNAMICS
  case 1: return 31;                             // GB_DYNAMICS
  case 2: return 0;                              // GENERAL_MINIMIZATION
  case 3: return 24;                             // GB_MINIMIZATION
  case 4: return 7 | (cache_depth << 8);         // LANGEVIN_DYNAMICS
  case 5: return 31 | (cache_depth << 8);        // GB_LANGEVIN_DYNAMICS
  case 6: return 0;                              // NONE
  default: break;
  }
  throw Error(SB_ERR_ARGUMENT, "unknown initialization task " + std::to_string(task));
}

void distributeRefresh(std::vector<WorkUnit>* wus, int natom, int code) {
  const int nwu = static_cast<int>(wus->size());
  if (code == 0) {
    return;
  }
  int tasks = 0;
  for (int b = 0; b < 8; b++) {
    tasks += (code >> b) & 1;
  }
  const int blocks = (natom + kRefreshBlock - 1) / kRefreshBlock;
  tasks += ((code >> 8) > 0) ? 1 : 0;
  auto assign = [&](int w, int first, int count, int work) {
    if (w >= nwu) {
      throw Error(SB_ERR_ARGUMENT, "more refresh assignments than work units");
    }
    (*wus)[w].refresh_start = first;
    (*wus)[w].refresh_code = work | (count << 16);
  };
  if (tasks * blocks < nwu) {
    int w = 0;
    if ((code & 0xff00) > 0) {
      for (int a = 0; a < natom; a += kRefreshBlock) {
        assign(w++, a, std::min(kRefreshBlock, natom - a), code & 0xff00);
      }
    }
    for (int b = 0; b < 8; b++) {
      if ((code >> b) & 1) {
        for (int a = 0; a < natom; a += kRefreshBlock) {
          assign(w++, a, std::min(kRefreshBlock, natom - a), 1 << b);
        }
      }
    }
  }
  else if ((code & 0xffff) > 0) {
    const int per_wu = std::max((blocks + nwu - 1) / nwu, 1) * kRefreshBlock;
    int w = 0;
    for (int a = 0; a < natom; a += per_wu) {
      assign(w++, a, std::min(per_wu, natom - a), code & 0xffff);
    }
  }
}

struct WorkUnitTables {
  std::vector<int> abstracts;
  std::vector<uint32_t> instructions;
};

WorkUnitTables buildWorkUnits(const sb_topology* tops, int ntop, const int* topology_index,
                              int nsys, int task, int cache_depth) {
  const MaskSynthesis ms = buildSynthesis(tops, ntop, topology_index, nsys);
  long long tiles_all = 0;
  for (int s = 0; s < nsys; s++) {
    const long long e = (ms.atom_counts[s] + kTileLen - 1) / kTileLen;
    tiles_all += e * (e + 1) / 2;
  }
  const int targets[4] = {8, 16, 32, 64};
  const long long caps[4] = {2048, 4096, 8192, 131072};
  int target = 0;
  for (int k = 0; k < 4 && target == 0; k++) {
    if ((tiles_all + targets[k] - 1) / targets[k] < caps[k]) {
      target = targets[k];
    }
  }
  if (target == 0) {
    throw Error(SB_ERR_UNSUPPORTED, "syntheses needing STORMM's 256-tile work units are not "
                "reproduced");
  }
  std::vector<WorkUnit> wus = enumerateWorkUnits(ms, target);
  const int padded_natom = ms.atom_offsets.back() + ((ms.atom_counts.back() + 31) / 32) * 32;
  distributeRefresh(&wus, padded_natom, initializationCode(task, cache_depth));
  WorkUnitTables out;
  out.abstracts.assign(wus.size() * kAbstractLength, -1);
  int insr = 0;
  for (size_t w = 0; w < wus.size(); w++) {
    const WorkUnit &wu = wus[w];
    int* a = &out.abstracts[w * kAbstractLength];
    const int nt = static_cast<int>(wu.tiles.size());
    a[0] = wu.import_count;
    for (int i = 0; i < wu.import_count; i++) {
      a[1 + i] = wu.imports[i];
      a[kMaxImports + 8 + i] = wu.import_sys[i];
    }
    for (int i = 0; i < kMaxImports / 4; i++) {
      a[1 + kMaxImports + i] = wu.size_keys[i];
    }
    a[kMaxImports + 6] = insr;
    a[kMaxImports + 7] = insr + nt;
    a[2 * kMaxImports + 8] = wu.init_mask;
    a[2 * kMaxImports + 9] = wu.refresh_start;
    a[2 * kMaxImports + 10] = wu.refresh_code;
    const int padded = ((nt + 31) / 32) * 32;
    for (int k = 0; k < padded; k++) {
      out.instructions.push_back(k < nt ? wu.insr_x[k] : 0u);
      out.instructions.push_back(k < nt ? wu.insr_y[k] : 0u);
    }
    insr += padded;
  }
  return out;
}

}  // namespace

}  // namespace sb

extern "C" int sb_static_exclusion_mask_synthesis(const sb_topology* tops, int ntop,
                                                  const int* topology_index, int nsys,
                                                  int* supertile_map_bounds,
                                                  int* supertile_map_idx,
                                                  long long* n_supertile_map, int* tile_map_idx,
                                                  long long* n_tile_map, uint32_t* mask_data,
                                                  long long* n_mask_data) {
  try {
    sb::checkSynthesisArgs(tops, ntop, topology_index, nsys);
    const sb::MaskSynthesis ms = sb::buildSynthesis(tops, ntop, topology_index, nsys);
    if (supertile_map_bounds != nullptr) {
      std::copy(ms.super_bounds.begin(), ms.super_bounds.end(), supertile_map_bounds);
    }
    sb::deliver(ms.super_map, supertile_map_idx, n_supertile_map, "the supertile map");
    sb::deliver(ms.tile_map, tile_map_idx, n_tile_map, "the tile map");
    sb::deliver(ms.masks, mask_data, n_mask_data, "the mask data");
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

extern "C" int sb_nonbonded_work_units(const sb_topology* tops, int ntop,
                                       const int* topology_index, int nsys, int init_task,
                                       int random_cache_depth, int* abstracts,
                                       long long* n_abstracts, uint32_t* instructions,
                                       long long* n_instructions) {
  try {
    sb::checkSynthesisArgs(tops, ntop, topology_index, nsys);
    const sb::WorkUnitTables wt = sb::buildWorkUnits(tops, ntop, topology_index, nsys, init_task,
                                                     random_cache_depth);
    sb::deliver(wt.abstracts, abstracts, n_abstracts, "the work-unit abstracts");
    sb::deliver(wt.instructions, instructions, n_instructions, "the tile instructions");
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
