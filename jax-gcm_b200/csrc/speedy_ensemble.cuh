// speedy_ensemble.cuh -- what the batched forward and the batched adjoint share: the tile
// list over ragged members, the per-class constants passed by value, and the adjoint's
// cloud-top pre-pass over all tiles (each member's level set and per-latitude solar table;
// the forward forms both in its first launch).
#pragma once

#include <algorithm>
#include <vector>

#include "speedy_kernels.cuh"

namespace spd {

// Level-set state of a member in the forward: S points at its accumulator T of the true level
// set; R (S[ls_stride]) is its redo flag and P (S[2 ls_stride]) the level set its last forward
// used, which the next forward predicts.
enum { LS_T = 0, LS_R = 1, LS_P = 2 };
// Words of one forward launch (TileSource::launch): the count of blocks done, whether any member
// must be redone, and (cumulative, in the region's last 16 bytes) the members redone so far.
enum { LW_DONE = 0, LW_ANY = 1 };

struct MemberDev {
  spd_inputs_t in;
  spd_outputs_t out;
  int C, il, kx, cls;
  uint32_t* S;
  int ls_stride, reserved;
};

struct ClassArgs {
  ConstsD cls[SPD_MAX_CLASSES];
};

struct Tile {
  int member, col0;
};

// Where a forward launch takes its tiles from: a plan's member table and tile list, or (when
// `members` is null) the one member given by value, whose tile t covers columns
// t*kNT .. t*kNT + kNT - 1.  Passed by value to the kernels.
struct TileSource {
  const MemberDev* members;
  const Tile* tiles;
  MemberDev single;
  int nmembers;
  uint32_t* launch;   // the launch words
  uint32_t* redone;   // cumulative count of members redone
};

// The member of tile t, copied: the kernels read its field pointers from the copy, which no
// store to an output field can alias (a reference into the plan would make the compiler reload
// the pointers after every store).
__device__ __forceinline__ MemberDev tile_member(const TileSource& T, int t, int& col0) {
  if (T.members == nullptr) {
    col0 = t * kNT;
    return T.single;
  }
  const Tile tl = T.tiles[t];
  col0 = tl.col0;
  return T.members[tl.member];
}

// Prefetches into L2 the `nrows` rows of a full tile (row(r): the first float of row r, 128
// consecutive floats), one prefetch per 128-byte line, spread over the block's threads.
template <class RowFn>
__device__ __forceinline__ void prefetch_tile_rows(int nrows, RowFn row) {
  static_assert(kNT == 128, "a tile row is four 128-byte lines");
  for (int i = threadIdx.x; i < nrows * 4; i += kNT) {
    const float* p = row(i >> 2) + (i & 3) * 32;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

// The forward (speedy_ensemble.cu) over the ntiles tiles, after clearing the launch words and
// every member's T and R (clear_bytes from T.launch).  speculate: the fused launch uses each
// member's predicted level set P and a fixup launch redoes the members whose prediction missed;
// otherwise a level-set launch forms every T before the fused launch reads it.  grid_blocks:
// 0 = persistent grids of SMs x resident blocks; > 0 = the fused launch's persistent grid;
// SPD_GRID_PER_TILE = one block per tile.  kx_layout is the largest level count among the
// tiles (it sizes the fused launch's shared-memory arena).
int launch_forward(const ClassArgs& A, const TileSource& T, int ntiles, int kx_layout,
                   int grid_blocks, bool speculate, size_t clear_bytes, cudaStream_t st,
                   cudaEvent_t marker);

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// M: any member record with in, C, il, kx, cls, S and table.
template <int KX, class M>
__device__ __forceinline__ void prepass_tile(const ClassArgs& A, const M& m, int c) {
  const Consts& K = A.cls[m.cls].K;
  if (c < m.il) m.table[c] = zonal_row(K.tyear, __ldg(m.in.sia + c), __ldg(m.in.coa + c));
  const uint32_t bit = (c < m.C) ? prepass_column<KX>(K, m.in, c, m.C) : 0u;
  or_level_set(bit, m.S);
}

template <class M>
__device__ __forceinline__ void prepass_tiles(const ClassArgs& A, const M* __restrict__ members,
                                              const Tile* __restrict__ tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const M& m = members[tl.member];
    const int c = tl.col0 + threadIdx.x;
    switch (m.kx) {  // uniform per block
      case 16: prepass_tile<16>(A, m, c); break;
      case 8: prepass_tile<8>(A, m, c); break;
      default: prepass_tile<7>(A, m, c); break;
    }
  }
}

// Device plan layout: header, member records, tile list, level-set region, solar tables.  The
// level-set region: 16 bytes of launch words, then nw words each of every member's T, R and P
// (nw = member count rounded up to 4), then 16 bytes whose first word counts the members the
// forward redid (its prediction missed).
struct PlanLayout {
  size_t members, tiles, levelset, tables, total;
  int ntiles, nw;
};

inline size_t levelset_region_bytes(int nw) { return 16 + 12 * (size_t)nw + 16; }

// HM: host member description with ix and il.
template <class HM>
inline PlanLayout plan_layout(const HM* members, int n, size_t record_bytes) {
  PlanLayout L;
  int ntiles = 0;
  size_t tab = 0;
  for (int i = 0; i < n; ++i) {
    const int C = members[i].ix * members[i].il;
    ntiles += (C + kNT - 1) / kNT;
    tab += align256((size_t)members[i].il * sizeof(ZonalRow));
  }
  L.ntiles = ntiles;
  L.members = 256;
  L.tiles = L.members + align256((size_t)n * record_bytes);
  L.nw = (n + 3) & ~3;
  L.levelset = L.tiles + align256((size_t)ntiles * sizeof(Tile));
  L.tables = L.levelset + align256(levelset_region_bytes(L.nw));
  L.total = L.tables + tab;
  return L;
}

// The members' T words (device address) in a plan at dbase.
inline uint32_t* levelset_T(const PlanLayout& L, char* dbase) {
  return reinterpret_cast<uint32_t*>(dbase + L.levelset + 16);
}

// The tile list: tiles of 16-level members first, then fewer levels (heavier work first).
// Returns the tile count.  DM: device member record with C and kx.
template <class DM>
inline int plan_tile_list(const DM* md, int n, Tile* tl) {
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return md[a].kx > md[b].kx; });
  int t = 0;
  for (int i : order)
    for (int c0 = 0; c0 < md[i].C; c0 += kNT) tl[t++] = Tile{i, c0};
  return t;
}

// Fills each record's level-set and table pointers (device addresses) and the tile list:
// tiles of 16-level members first, then fewer levels (heavier work first).  Returns the tile
// count.  DM: device member record with C, il, kx, S and table.
template <class DM>
inline int plan_tiles(DM* md, int n, const PlanLayout& L, char* dbase, Tile* tl) {
  size_t tab = L.tables;
  for (int i = 0; i < n; ++i) {
    md[i].S = levelset_T(L, dbase) + i;
    md[i].table = reinterpret_cast<ZonalRow*>(dbase + tab);
    tab += align256((size_t)md[i].il * sizeof(ZonalRow));
  }
  return plan_tile_list(md, n, tl);
}

}  // namespace spd
