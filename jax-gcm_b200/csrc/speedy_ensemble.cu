// speedy_ensemble.cu -- the batched ragged ensemble: many members of mixed resolution and
// level count in two persistent launches over one tile list.
//
// A member is one grid instance (its own arrays, ix*il columns, kx levels).  The plan splits
// every member into tiles of kNT consecutive columns (a tile never straddles members), ordered
// by level count (16-level tiles first, the heavier work), and keeps per member the field
// pointers and its cloud-top level-set words (P: the prediction, T: the true set, R: missed).
// The one cross-column dependency is the level set S (shortwave_radiation.py:62-68).  Two
// launch forms:
//   speculating (the default): the fused launch runs every column whole, in one pass, with
//     each member's predicted set P (the previous call's) while the columns OR their own cloud
//     tops into T; its last block compares T with P and marks the members that missed (R).
//     The fixup launch, a programmatic dependent launch of one resident wave, computes the
//     missed members again with their true set; when none missed its blocks read one word
//     and return.
//   level set first (accumulating calls, which must not add a column's diagnostics twice, and
//     calls that ask for no prediction): a light launch forms every member's S from the
//     cloud-top part of every column, then the fused launch reads it.
// The launches are persistent or one block per tile (gridDim blocks stride over the tile
// list).  The plain per-instance forward (spd_fwd) runs the same kernels over a one-member
// plan given by value, so that the two paths agree bitwise.
// Constants shared by a class of members (kx, date, switches, vertical grid, parameters) travel
// by value in the kernel parameters.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "speedy_ensemble.cuh"

namespace spd {

int check_forward_instance(const spd_desc_t* d, const spd_inputs_t* in,
                           const spd_outputs_t* out);
Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p);

// Rows the level-set launch reads for a tile of member m: T, q, phi at every level, psa.
__device__ __forceinline__ void prefetch_levelset_tile(const MemberDev& m, int col0) {
  const int kx = m.kx;
  const size_t C = m.C;
  prefetch_tile_rows(3 * kx + 1, [&](int r) -> const float* {
    if (r < kx) return m.in.temperature + r * C + col0;
    if (r < 2 * kx) return m.in.specific_humidity + (r - kx) * C + col0;
    if (r < 3 * kx) return m.in.geopotential + (r - 2 * kx) * C + col0;
    return m.in.normalized_surface_pressure + col0;
  });
}

// The tile this block processes `stride` tiles ahead, if it is a full tile: its rows are
// prefetched into L2 while the current tile computes.
template <class F>
__device__ __forceinline__ void prefetch_ahead(const TileSource& T, int t, int stride, int ntiles,
                                               F prefetch) {
  const int tn = t + stride;
  if (stride <= 0 || tn >= ntiles) return;
  int col0n;
  const MemberDev mn = tile_member(T, tn, col0n);
  if (mn.C - col0n >= kNT) prefetch(mn, col0n);
}

// Level-set launch (when the forward does not speculate): every member's cloud-top level set
// T, an OR over its columns' clipped cloud tops, formed by the first half's top-only form.
__global__ void __launch_bounds__(kNT, 5) ensemble_levelset(const __grid_constant__ ClassArgs A,
                                                            const __grid_constant__ TileSource T,
                                                            int ntiles, int pf_stride) {
  // the fused launch may start as this one's blocks retire (it waits for completion before
  // reading anything written here)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int col0;
    const MemberDev m = tile_member(T, t, col0);
    const int c = col0 + threadIdx.x;
    const ConstsD& CD = A.cls[m.cls];
    prefetch_ahead(T, t, pf_stride, ntiles, prefetch_levelset_tile);
    uint32_t bit = 0;
    if (c < m.C) {
      switch (m.kx) {  // uniform per block
        case 16: bit = levelset_bit<16>(CD, m.in, c, m.C); break;
        case 8: bit = levelset_bit<8>(CD, m.in, c, m.C); break;
        default: bit = levelset_bit<7>(CD, m.in, c, m.C); break;
      }
    }
    or_level_set(bit, m.S + LS_T * m.ls_stride);
  }
}

template <int KX>
__device__ __forceinline__ uint32_t fused_column(const ConstsD& CD, float* sm,
                                                 const MemberDev& m, const uint32_t* S, int c) {
  return fused_process<KX>(CD, sm, m.in, m.out, S, c, m.C, m.il);
}

// The end of a fused launch, in its last block to finish: every member's P becomes the level
// set its columns formed (T); when speculating, R marks the members whose prediction P missed,
// the launch word ANY says whether any did, and the cumulative count grows by their number.
// `words` are two words of the block's shared memory that the columns no longer use (the
// fused launch declares no static shared memory: one more word would leave room for three
// blocks per SM instead of four at 16 levels).
__device__ __forceinline__ void finish_fused(const TileSource& T, bool speculate,
                                             uint32_t* words) {
  uint32_t& last = words[0];
  uint32_t& redo_block = words[1];
  __syncthreads();  // every warp of this block has issued its level-set ORs and left the arena
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(T.launch + LW_DONE, 1u) == gridDim.x - 1;
    redo_block = 0;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nm = T.members ? T.nmembers : 1;
  uint32_t redo = 0;
  for (int i = threadIdx.x; i < nm; i += blockDim.x) {
    const MemberDev& m = T.members ? T.members[i] : T.single;
    volatile uint32_t* S = m.S;
    const uint32_t t = S[LS_T * m.ls_stride];
    if (speculate) {
      const uint32_t r = t != S[LS_P * m.ls_stride] ? 1u : 0u;
      S[LS_R * m.ls_stride] = r;
      redo += r;
    }
    S[LS_P * m.ls_stride] = t;
  }
  if (redo) atomicAdd(&redo_block, redo);
  __syncthreads();
  if (threadIdx.x == 0) {
    T.launch[LW_ANY] = redo_block ? 1u : 0u;
    if (redo_block) atomicAdd(T.redone, redo_block);
  }
}

// Fused launch: every column whole (fused_process).  speculate = 1: the shortwave uses each
// member's predicted level set P while the columns OR their own cloud tops into T; else T is
// complete (the level-set launch formed it) and the columns read it.
__global__ void __launch_bounds__(kNT, 4) ensemble_fused(const __grid_constant__ ClassArgs A,
                                                         const __grid_constant__ TileSource T,
                                                         int ntiles, int speculate) {
  extern __shared__ float sm[];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int col0;
    const MemberDev m = tile_member(T, t, col0);
    const int c = col0 + threadIdx.x;
    const uint32_t* S = m.S + (speculate ? LS_P : LS_T) * m.ls_stride;
    uint32_t bit = 0;
    if (c < m.C) {
      const ConstsD& CD = A.cls[m.cls];
      switch (m.kx) {
        case 16: bit = fused_column<16>(CD, sm, m, S, c); break;
        case 8: bit = fused_column<8>(CD, sm, m, S, c); break;
        default: bit = fused_column<7>(CD, sm, m, S, c); break;
      }
    }
    if (speculate) or_level_set_warp(bit, m.S + LS_T * m.ls_stride);
  }
  // the fixup launch may start as this one's blocks retire; it waits for completion
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  finish_fused(T, speculate != 0, reinterpret_cast<uint32_t*>(sm));
}

// Fixup launch after a speculating fused launch: the members whose prediction missed (R set)
// are computed again with their true level set (P, now equal to T).  In the common case no
// member missed and every block returns after reading one word.
__global__ void __launch_bounds__(kNT, 4) ensemble_fixup(const __grid_constant__ ClassArgs A,
                                                         const __grid_constant__ TileSource T,
                                                         int ntiles) {
  extern __shared__ float sm[];
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (*reinterpret_cast<volatile uint32_t*>(T.launch + LW_ANY) == 0u) return;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int col0;
    const MemberDev m = tile_member(T, t, col0);
    if (*reinterpret_cast<volatile uint32_t*>(m.S + LS_R * m.ls_stride) == 0u) continue;
    const int c = col0 + threadIdx.x;
    const uint32_t* S = m.S + LS_P * m.ls_stride;
    if (c < m.C) {
      const ConstsD& CD = A.cls[m.cls];
      switch (m.kx) {
        case 16: fused_column<16>(CD, sm, m, S, c); break;
        case 8: fused_column<8>(CD, sm, m, S, c); break;
        default: fused_column<7>(CD, sm, m, S, c); break;
      }
    }
  }
}

static size_t arena_bytes(int kx) { return (size_t)kNumArrays * kx * kNT * sizeof(float); }

namespace {
struct Residency {
  int sms = 0, lvl = 0, cols[17] = {};  // resident blocks per SM (level-set launch;
                                          // fused launch by arena level count)
};

// SMs and resident blocks per SM of both kernels on the current device, set up once per device
// (the shared-memory attribute of a kernel is a per-device setting).
int residency(Residency& R) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static Residency cached[kMaxDevices];
  static bool done[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SPD_ERR_CUDA;
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    Residency r;
    if (cudaFuncSetAttribute(ensemble_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes<16>()) != cudaSuccess ||
        cudaFuncSetAttribute(ensemble_fixup, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes<16>()) != cudaSuccess ||
        cudaDeviceGetAttribute(&r.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r.lvl, ensemble_levelset, kNT, 0) !=
            cudaSuccess)
      return SPD_ERR_CUDA;
    for (int kx : {7, 8, 16})
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r.cols[kx], ensemble_fused, kNT,
                                                        arena_bytes(kx)) != cudaSuccess)
        return SPD_ERR_CUDA;
    r.lvl = std::max(r.lvl, 1);
    for (int kx : {7, 8, 16}) r.cols[kx] = std::max(r.cols[kx], 1);
    cached[dev] = r;
    done[dev] = true;
  }
  R = cached[dev];
  return SPD_OK;
}
}  // namespace

// Launches kernel<<<grid, kNT, smem, st>>>(args...) as a programmatic dependent launch: its
// blocks may start as the previous launch's blocks retire (they wait on the device,
// griddepcontrol.wait, before reading what that launch writes).
template <class... KArgs, class... Args>
static int launch_dependent(void (*kernel)(KArgs...), int grid, size_t smem, cudaStream_t st,
                            Args... args) {
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kNT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, kernel, args...) != cudaSuccess) return SPD_ERR_CUDA;
  return SPD_OK;
}

int launch_forward(const ClassArgs& A, const TileSource& T, int ntiles, int kx_layout,
                   int grid_blocks, bool speculate, size_t clear_bytes, cudaStream_t st,
                   cudaEvent_t marker) {
  Residency R;
  const int rc = residency(R);
  if (rc != SPD_OK) return rc;
  const int res_lvl = R.sms * R.lvl, res_cols = R.sms * R.cols[kx_layout];
  int grid_lvl, grid_cols, pf_lvl;
  if (grid_blocks == SPD_GRID_PER_TILE) {
    // one block per tile; the blocks resident beside this one run the next wave, so the tile
    // a wave ahead is the one to prefetch
    grid_lvl = grid_cols = ntiles;
    pf_lvl = res_lvl;
  } else {
    grid_lvl = std::min(res_lvl, ntiles);
    grid_cols = std::min(grid_blocks > 0 ? grid_blocks : res_cols, ntiles);
    pf_lvl = grid_lvl;
  }
  const size_t arena = arena_bytes(kx_layout);
  // the fixup is one resident wave striding over the tiles: its blocks read one word and return
  // when no prediction missed, and a grid of one block per tile spends microseconds on
  // scheduling thousands of such blocks
  const int grid_fix = std::min(grid_cols, res_cols);
  // the launch words and every member's T and R start at zero; P is kept from the last call
  if (cudaMemsetAsync(T.launch, 0, clear_bytes, st) != cudaSuccess) return SPD_ERR_CUDA;
  int r;
  if (speculate) {
    ensemble_fused<<<grid_cols, kNT, arena, st>>>(A, T, ntiles, 1);
    if (marker) {  // timing hook: the fused launch apart, then the fixup in plain stream order
      if (cudaEventRecord(marker, st) != cudaSuccess) return SPD_ERR_CUDA;
      ensemble_fixup<<<grid_fix, kNT, arena, st>>>(A, T, ntiles);
      r = SPD_OK;
    } else {
      r = launch_dependent(ensemble_fixup, grid_fix, arena, st, A, T, ntiles);
    }
  } else {
    ensemble_levelset<<<grid_lvl, kNT, 0, st>>>(A, T, ntiles, pf_lvl);
    if (marker) {  // timing hook: the two launches apart, in plain stream order
      if (cudaEventRecord(marker, st) != cudaSuccess) return SPD_ERR_CUDA;
      ensemble_fused<<<grid_cols, kNT, arena, st>>>(A, T, ntiles, 0);
      r = SPD_OK;
    } else {
      r = launch_dependent(ensemble_fused, grid_cols, arena, st, A, T, ntiles, 0);
    }
  }
  if (r != SPD_OK) return r;
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}

int preload_ensemble() {
  cudaFuncAttributes a;
  bool ok = cudaFuncGetAttributes(&a, ensemble_levelset) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_fused) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_fixup) == cudaSuccess;
  return ok ? SPD_OK : SPD_ERR_CUDA;
}

}  // namespace spd

extern "C" {

size_t spd_ensemble_plan_bytes(const spd_member_t* members, int nmembers) {
  if (!members || nmembers <= 0) return 0;
  return spd::plan_layout(members, nmembers, sizeof(spd::MemberDev)).total;
}

int spd_ensemble_plan(const spd_class_t* classes, int nclasses, const spd_member_t* members,
                      int nmembers, void* plan_host, void* plan_device, size_t plan_bytes,
                      spd_plan_info_t* info) {
  using namespace spd;
  if (!classes || !members || !plan_host || !plan_device || !info) return SPD_ERR_NULL;
  if (nclasses <= 0 || nclasses > SPD_MAX_CLASSES || nmembers <= 0) return SPD_ERR_SHAPE;
  if (reinterpret_cast<uintptr_t>(plan_device) & 255u) return SPD_ERR_SCRATCH;
  const PlanLayout L = plan_layout(members, nmembers, sizeof(MemberDev));
  if (plan_bytes < L.total) return SPD_ERR_SCRATCH;
  for (int i = 0; i < nmembers; ++i) {
    const spd_member_t& m = members[i];
    if (m.cls < 0 || m.cls >= nclasses) return SPD_ERR_SHAPE;
    spd_desc_t d = classes[m.cls].desc;
    d.ix = m.ix;
    d.il = m.il;
    const int rc = check_forward_instance(&d, &m.in, &m.out);
    if (rc != SPD_OK) return rc;
  }
  char* h = static_cast<char*>(plan_host);
  char* dbase = static_cast<char*>(plan_device);
  memset(h, 0, L.total);
  MemberDev* md = reinterpret_cast<MemberDev*>(h + L.members);
  for (int i = 0; i < nmembers; ++i) {
    const spd_member_t& m = members[i];
    md[i].in = m.in;
    md[i].out = m.out;
    md[i].C = m.ix * m.il;
    md[i].il = m.il;
    md[i].kx = classes[m.cls].desc.kx;
    md[i].cls = m.cls;
  }
  for (int i = 0; i < nmembers; ++i) {
    md[i].S = levelset_T(L, dbase) + i;
    md[i].ls_stride = L.nw;
  }
  const int t = plan_tile_list(md, nmembers, reinterpret_cast<Tile*>(h + L.tiles));
  info->nmembers = nmembers;
  info->ntiles = t;
  info->levelset_offset = L.levelset;
  info->levelset_bytes = levelset_region_bytes(L.nw);
  info->plan_bytes = L.total;
  return SPD_OK;
}

int spd_ensemble_fwd(const spd_class_t* classes, int nclasses, void* plan_device,
                     const spd_plan_info_t* info, int grid_blocks, void* stream) {
  return spd_ensemble_fwd_marked(classes, nclasses, plan_device, info, grid_blocks, stream,
                                 nullptr);
}

int spd_ensemble_fwd_marked(const spd_class_t* classes, int nclasses, void* plan_device,
                            const spd_plan_info_t* info, int grid_blocks, void* stream,
                            void* event) {
  using namespace spd;
  if (!classes || !plan_device || !info) return SPD_ERR_NULL;
  if (nclasses <= 0 || nclasses > SPD_MAX_CLASSES || info->ntiles <= 0) return SPD_ERR_SHAPE;
  if (grid_blocks < 0 && grid_blocks != SPD_GRID_PER_TILE) return SPD_ERR_SHAPE;
  ClassArgs A;
  int kx_layout = 0;
  for (int i = 0; i < nclasses; ++i) {
    A.cls[i].K = make_consts(&classes[i].desc, &classes[i].vgrid, &classes[i].params);
    A.cls[i].D = derive_constants(&classes[i].desc, &classes[i].vgrid, &classes[i].params);
    kx_layout = std::max(kx_layout, classes[i].desc.kx);
  }
  if (kx_layout != 7 && kx_layout != 8 && kx_layout != 16) return SPD_ERR_KX;
  char* base = static_cast<char*>(plan_device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  bool speculate = true;
  for (int i = 0; i < nclasses; ++i)
    if (classes[i].desc.flags & (SPD_ACCUMULATE_DIAGNOSTICS | SPD_NO_SPECULATION))
      speculate = false;
  const int nw = (info->nmembers + 3) & ~3;
  TileSource T{};
  T.members = reinterpret_cast<const MemberDev*>(base + 256);
  T.tiles = reinterpret_cast<const Tile*>(
      base + 256 + align256((size_t)info->nmembers * sizeof(MemberDev)));
  T.nmembers = info->nmembers;
  T.launch = reinterpret_cast<uint32_t*>(base + info->levelset_offset);
  T.redone = T.launch + (16 + 12 * (size_t)nw) / sizeof(uint32_t);
  return launch_forward(A, T, info->ntiles, kx_layout, grid_blocks, speculate,
                        16 + 8 * (size_t)nw, st, static_cast<cudaEvent_t>(event));
}

}  // extern "C"
