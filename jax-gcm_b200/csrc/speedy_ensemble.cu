// speedy_ensemble.cu -- the batched ragged ensemble: many members of mixed resolution and
// level count in two persistent launches over one tile list.
//
// A member is one grid instance (its own arrays, ix*il columns, kx levels).  The plan splits
// every member into tiles of kNT consecutive columns (a tile never straddles members), ordered
// by level count (16-level tiles first, the heavier work), and keeps per member the field
// pointers, its cloud-top level-set word and its per-latitude solar table.  Launch 1 (light)
// forms each member's level set S and solar table from the cloud-top part of every column;
// launch 2 runs every column whole, in one pass, reading its member's S (the one cross-column
// dependency, shortwave_radiation.py:62-68) and solar table.  Both launches are persistent:
// gridDim blocks stride over the tile list.  The plain per-instance forward (spd_fwd) runs the
// same two kernels over a one-member plan given by value, so that the two paths agree bitwise.
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

// Launch 1: every member's per-latitude solar table and cloud-top level set S (an OR over its
// columns' clipped cloud tops, formed by the first half's top-only form).
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
    if (c < m.il) m.table[c] = zonal_row(CD.K.tyear, __ldg(m.in.sia + c), __ldg(m.in.coa + c));
    uint32_t bit = 0;
    if (c < m.C) {
      switch (m.kx) {  // uniform per block
        case 16: bit = levelset_bit<16>(CD, m.in, c, m.C); break;
        case 8: bit = levelset_bit<8>(CD, m.in, c, m.C); break;
        default: bit = levelset_bit<7>(CD, m.in, c, m.C); break;
      }
    }
    or_level_set(bit, m.S);
  }
}

// Launch 2: every column whole (fused_process), reading its member's S and solar table.
__global__ void __launch_bounds__(kNT, 4) ensemble_fused(const __grid_constant__ ClassArgs A,
                                                         const __grid_constant__ TileSource T,
                                                         int ntiles) {
  extern __shared__ float sm[];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int col0;
    const MemberDev m = tile_member(T, t, col0);
    const int c = col0 + threadIdx.x;
    if (c < m.C) {
      const ConstsD& CD = A.cls[m.cls];
      switch (m.kx) {
        case 16: fused_process<16>(CD, sm, m.in, m.out, m.S, m.table, c, m.C, m.il); break;
        case 8: fused_process<8>(CD, sm, m.in, m.out, m.S, m.table, c, m.C, m.il); break;
        default: fused_process<7>(CD, sm, m.in, m.out, m.S, m.table, c, m.C, m.il); break;
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

int launch_forward(const ClassArgs& A, const TileSource& T, int ntiles, int kx_layout,
                   int grid_blocks, cudaStream_t st, cudaEvent_t marker) {
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
  ensemble_levelset<<<grid_lvl, kNT, 0, st>>>(A, T, ntiles, pf_lvl);
  if (marker) {  // timing hook: the two launches apart, in plain stream order
    if (cudaEventRecord(marker, st) != cudaSuccess) return SPD_ERR_CUDA;
    ensemble_fused<<<grid_cols, kNT, arena_bytes(kx_layout), st>>>(A, T, ntiles);
    return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
  }
  // programmatic dependent launch: the second launch's blocks take SMs as the first launch's
  // blocks retire and load their inputs, then wait (griddepcontrol.wait) for its completion
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_cols);
  cfg.blockDim = dim3(kNT);
  cfg.dynamicSmemBytes = arena_bytes(kx_layout);
  cfg.stream = st;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, ensemble_fused, A, T, ntiles) != cudaSuccess) return SPD_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}

int preload_ensemble() {
  cudaFuncAttributes a;
  bool ok = cudaFuncGetAttributes(&a, ensemble_levelset) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_fused) == cudaSuccess;
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
  const int t = plan_tiles(md, nmembers, L, dbase, reinterpret_cast<Tile*>(h + L.tiles));
  info->nmembers = nmembers;
  info->ntiles = t;
  info->levelset_offset = L.levelset;
  info->levelset_bytes = align256((size_t)nmembers * sizeof(uint32_t));
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
  TileSource T{};
  T.members = reinterpret_cast<const MemberDev*>(base + 256);
  T.tiles = reinterpret_cast<const Tile*>(
      base + 256 + align256((size_t)info->nmembers * sizeof(MemberDev)));
  if (cudaMemsetAsync(base + info->levelset_offset, 0, info->levelset_bytes, st) != cudaSuccess)
    return SPD_ERR_CUDA;
  return launch_forward(A, T, info->ntiles, kx_layout, grid_blocks, st,
                        static_cast<cudaEvent_t>(event));
}

}  // extern "C"
