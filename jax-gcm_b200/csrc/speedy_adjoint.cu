// speedy_adjoint.cu -- the adjoint of the forward: one instance (spd_vjp) or a ragged ensemble
// of them (spd_ensemble_vjp), both through the same two kernels.
//
// Launch 1 is the forward's cloud-top pre-pass over the tile list of speedy_ensemble.cuh (each
// member's level set S and per-latitude solar table: neither carries a derivative).  Launch 2
// runs one thread per column, one block per tile: the hand-written reverse pass of speedy_vjp.h
// recomputes the column's forward and walks its terms backwards, writing the state gradients;
// the 12 parameter gradients are summed per thread, then per block, then added to the tile's
// member with one atomicAdd per parameter.  A single instance is a one-member plan written
// into its scratch by a small kernel, so it runs exactly the ensemble's instructions.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string.h>

#include <algorithm>

#include "speedy_ensemble.cuh"
#include "speedy_vjp.h"

namespace spd {

int check_instance(const spd_desc_t* d, const spd_inputs_t* in, const spd_outputs_t* out);
Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p);

constexpr int kAdjBlock = 128;

struct VjpArgs {
  spd_vgrid_t vg;
  spd_params_t p;
  uint32_t flags;
  int model_step, C, il;
  float ablco2, dt_seconds, q_tend_scale;
  float qcorv[SPD_MAX_KX], gamlat, pexp;  // orographic correction (SPD_OROGRAPHIC)
};

// One column's VJP: loads, the reverse pass, stores; adds the parameter gradients to pacc.
template <int KX>
__device__ __forceinline__ void vjp_column(const VjpArgs& A, const spd_inputs_t& in,
                                           const spd_cotangents_t& ct, const spd_grads_t& gr,
                                           uint32_t Sw, const ZonalRow* __restrict__ table,
                                           int c, int C, int il, float* pacc) {
  const spdvjp::Ctx x{&A.vg, &A.p, A.flags, A.model_step, Sw};
  spdgen::DiffParams<float> g;
  g.psmin = A.p.psmin; g.trcnv = A.p.trcnv; g.rhil = A.p.rhil; g.rhbl = A.p.rhbl;
  g.entmax = A.p.entmax; g.smf = A.p.smf; g.trlsc = A.p.trlsc; g.rhlsc = A.p.rhlsc;
  g.drhlsc = A.p.drhlsc; g.rhblsc = A.p.rhblsc; g.albcl = A.p.albcl; g.albcls = A.p.albcls;
  spdgen::ColumnIn<float, float> xi;
  float ct_t[KX], ct_q[KX];
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    xi.t[k] = __ldg(in.temperature + i);
    xi.q[k] = __ldg(in.specific_humidity + i);
    xi.phi[k] = __ldg(in.geopotential + i);
    ct_t[k] = __ldg(ct.temperature + i);
    ct_q[k] = __ldg(ct.specific_humidity + i);
  }
  const size_t lo = (size_t)(KX - 1) * C + c;
  xi.psa = __ldg(in.normalized_surface_pressure + c);
  xi.u_low = __ldg(in.u_wind + lo);
  xi.v_low = __ldg(in.v_wind + lo);
  xi.sst = __ldg(in.sea_surface_temperature + c);
  xi.stl = __ldg(in.stl_am + c);
  xi.soilw = __ldg(in.soilw_am + c);
  xi.snowc = __ldg(in.snowc_am + c);
  xi.sice = __ldg(in.sice_am + c);
  xi.alb0 = __ldg(in.alb0 + c);
  xi.fmask = __ldg(in.fmask + c);
  xi.orog = __ldg(in.orog + c);
  xi.phis0 = __ldg(in.phis0 + c);
  const ZonalRow z = table[c % il];
  xi.fsol = z.fsol; xi.ozupp = z.ozupp; xi.ozone = z.ozone; xi.zenit = z.zenit;
  xi.stratz = z.stratz; xi.sqrt_coa = z.sqrt_coa;
  spdvjp::Bar<KX, float> b;
  spdvjp::column_vjp<KX, float>(x, g, A.ablco2, A.dt_seconds, A.q_tend_scale, xi, ct_t, ct_q,
                                __ldg(ct.u_wind + lo), __ldg(ct.v_wind + lo), b, A.qcorv,
                                A.gamlat, A.pexp);
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    gr.temperature[i] = b.t[k];
    gr.specific_humidity[i] = b.q[k];
    gr.geopotential[i] = b.phi[k];
    gr.u_wind[i] = (k == KX - 1) ? b.u : 0.0f;
    gr.v_wind[i] = (k == KX - 1) ? b.v : 0.0f;
  }
  gr.normalized_surface_pressure[c] = b.psa;
#pragma unroll
  for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) pacc[j] += b.par[j];
}

// Sums pacc over the block and adds it to params with one atomic per parameter.  Every thread
// of the block must call it.
__device__ __forceinline__ void block_add_params(float* pacc, float* params) {
  __shared__ float red[kAdjBlock / 32][SPD_NUM_DIFF_PARAMS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) {
    float v = pacc[j];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < SPD_NUM_DIFF_PARAMS) {
    float v = 0.0f;
    for (int w = 0; w < kAdjBlock / 32; ++w) v += red[w][threadIdx.x];
    atomicAdd(params + threadIdx.x, v);
  }
  __syncthreads();
}

// ---- ensemble ----
struct VjpMemberDev {
  spd_inputs_t in;
  spd_cotangents_t ct;
  spd_grads_t gr;
  int C, il, kx, cls;
  uint32_t* S;
  ZonalRow* table;
};

struct VjpClassArgs {
  VjpArgs cls[SPD_MAX_CLASSES];
};

__global__ void __launch_bounds__(kBlock)
    ensemble_vjp_prepass(const __grid_constant__ ClassArgs A,
                         const VjpMemberDev* __restrict__ members,
                         const Tile* __restrict__ tiles, int ntiles) {
  // the adjoint launch accumulates each member's parameter gradients: zero them here
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    if (tl.col0 == 0 && threadIdx.x < SPD_NUM_DIFF_PARAMS)
      members[tl.member].gr.params[threadIdx.x] = 0.0f;
  }
  prepass_tiles(A, members, tiles, ntiles);
}

// Two register budgets of the same kernel: 128 registers for four blocks per SM, or 255 for two
// (1,376 against 2,088 bytes of stack, ptxas).  Two blocks per SM is the faster where every
// tile of the batch is resident at once (T85 with 16 levels, 256 tiles: 0.134 against
// 0.194 ms); four is the faster at T170 (1,024 tiles, 1.73 waves of four-per-SM residency
// against 3.46 of two).  The launch takes two per SM when the tiles fit in one such wave.  The
// translation unit is compiled without multiply-add contraction, so the two give the same bits
// (a member's gradients do not depend on the batch that carried it).
template <int kMinBlocks>
__global__ void __launch_bounds__(kAdjBlock, kMinBlocks)
    ensemble_adjoint(const __grid_constant__ VjpClassArgs A,
                     const VjpMemberDev* __restrict__ members, const Tile* __restrict__ tiles,
                     int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const VjpMemberDev& m = members[tl.member];
    const int c = tl.col0 + threadIdx.x;
    float pacc[SPD_NUM_DIFF_PARAMS];
#pragma unroll
    for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) pacc[j] = 0.0f;
    if (c < m.C) {
      const VjpArgs& V = A.cls[m.cls];
      const uint32_t Sw = *m.S;
      switch (m.kx) {  // uniform per block
        case 16: vjp_column<16>(V, m.in, m.ct, m.gr, Sw, m.table, c, m.C, m.il, pacc); break;
        case 8: vjp_column<8>(V, m.in, m.ct, m.gr, Sw, m.table, c, m.C, m.il, pacc); break;
        default: vjp_column<7>(V, m.in, m.ct, m.gr, Sw, m.table, c, m.C, m.il, pacc); break;
      }
    }
    block_add_params(pacc, m.gr.params);
  }
}

// The one-member plan of a single instance: its record and its tile list.
__global__ void __launch_bounds__(kBlock) vjp_single_plan(const VjpMemberDev rec,
                                                          VjpMemberDev* dst, Tile* tiles,
                                                          int ntiles) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) *dst = rec;
  for (; t < ntiles; t += gridDim.x * blockDim.x) tiles[t] = Tile{0, t * kNT};
}

struct OneMember {
  int ix, il;
};

inline PlanLayout single_layout(const spd_desc_t* d) {
  const OneMember m{d->ix, d->il};
  return plan_layout(&m, 1, sizeof(VjpMemberDev));
}

int preload_adjoint() {
  cudaFuncAttributes a;
  bool ok = true;
  ok &= cudaFuncGetAttributes(&a, vjp_single_plan) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_vjp_prepass) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_adjoint<4>) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, ensemble_adjoint<2>) == cudaSuccess;
  return ok ? SPD_OK : SPD_ERR_CUDA;
}

// Both launches over a plan already on the device (tiles at base + tiles_off).
static int launch_ensemble_vjp(const ClassArgs& P, const VjpClassArgs& V, char* base,
                               int nmembers, int ntiles, size_t levelset_offset,
                               size_t levelset_bytes, int grid_blocks, cudaStream_t st) {
  const VjpMemberDev* md = reinterpret_cast<const VjpMemberDev*>(base + 256);
  const size_t tiles_off = 256 + align256((size_t)nmembers * sizeof(VjpMemberDev));
  const Tile* tl = reinterpret_cast<const Tile*>(base + tiles_off);
  // Default: one block per tile.  The blocks are short (one tile's columns each), so the SMs
  // turn over often and a higher-priority stream's kernels (a forward batch) get them within
  // one block's time; a persistent grid would hold every SM until the whole batch is done.
  const int grid = grid_blocks > 0 ? std::min(grid_blocks, ntiles) : ntiles;
  const int grid_pre = std::min(ntiles, 65535);
  if (cudaMemsetAsync(base + levelset_offset, 0, levelset_bytes, st) != cudaSuccess)
    return SPD_ERR_CUDA;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return SPD_ERR_CUDA;
  ensemble_vjp_prepass<<<grid_pre, kBlock, 0, st>>>(P, md, tl, ntiles);
  if (grid <= 2 * sms)
    ensemble_adjoint<2><<<grid, kAdjBlock, 0, st>>>(V, md, tl, ntiles);
  else
    ensemble_adjoint<4><<<grid, kAdjBlock, 0, st>>>(V, md, tl, ntiles);
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}

static VjpArgs make_vjp_args(const spd_desc_t* desc, const spd_vgrid_t* vgrid,
                             const spd_params_t* params) {
  const Derived D = derive_constants(desc, vgrid, params);
  VjpArgs A;
  A.vg = *vgrid;
  A.p = *params;
  A.flags = desc->flags;
  A.model_step = desc->model_step;
  A.C = desc->ix * desc->il;
  A.il = desc->il;
  A.ablco2 = D.ablco2;
  A.dt_seconds = desc->dt_seconds;
  A.q_tend_scale = desc->q_tend_scale;
  for (int k = 0; k < SPD_MAX_KX; ++k) A.qcorv[k] = D.qcorv[k];
  A.gamlat = D.gamlat;
  A.pexp = D.pexp;
  return A;
}

// The fields spd_vjp reads and writes, validated like spd_fwd's.
static int check_vjp_member(const spd_desc_t* desc, const spd_inputs_t* in,
                            const spd_cotangents_t* ct, const spd_grads_t* grads) {
  if (!desc || !in || !ct || !grads) return SPD_ERR_NULL;
  spd_outputs_t dummy = {};
  float* probe = grads->temperature;
  dummy.u_wind = dummy.v_wind = dummy.temperature = dummy.specific_humidity = probe;
  dummy.precnv = dummy.precls = probe;
  int rc = check_instance(desc, in, &dummy);
  if (rc != SPD_OK) return rc;
  const void* req[] = {ct->u_wind, ct->v_wind, ct->temperature, ct->specific_humidity,
                       grads->u_wind, grads->v_wind, grads->specific_humidity,
                       grads->geopotential, grads->normalized_surface_pressure, grads->params};
  for (const void* p : req)
    if (!p) return SPD_ERR_NULL;
  return SPD_OK;
}

}  // namespace spd

extern "C" {

size_t spd_vjp_scratch_bytes(const spd_desc_t* desc) {
  if (!desc || desc->ix <= 0 || desc->il <= 0) return 0;
  return spd::single_layout(desc).total;
}

int spd_vjp(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
            const spd_inputs_t* in, const spd_cotangents_t* ct, const spd_grads_t* grads,
            void* scratch, size_t scratch_bytes, void* stream) {
  using namespace spd;
  if (!desc || !vgrid || !params || !in || !ct || !grads) return SPD_ERR_NULL;
  const int rc = check_vjp_member(desc, in, ct, grads);
  if (rc != SPD_OK) return rc;
  const PlanLayout L = single_layout(desc);
  if (!scratch || (reinterpret_cast<uintptr_t>(scratch) & 255u) || scratch_bytes < L.total)
    return SPD_ERR_SCRATCH;
  if (desc->kx != 7 && desc->kx != 8 && desc->kx != 16) return SPD_ERR_KX;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(scratch);
  ClassArgs P;
  VjpClassArgs V;
  P.cls[0].K = make_consts(desc, vgrid, params);
  P.cls[0].D = derive_constants(desc, vgrid, params);
  V.cls[0] = make_vjp_args(desc, vgrid, params);
  VjpMemberDev rec;
  rec.in = *in;
  rec.ct = *ct;
  rec.gr = *grads;
  rec.C = desc->ix * desc->il;
  rec.il = desc->il;
  rec.kx = desc->kx;
  rec.cls = 0;
  rec.S = reinterpret_cast<uint32_t*>(base + L.levelset);
  rec.table = reinterpret_cast<ZonalRow*>(base + L.tables);
  VjpMemberDev* dst = reinterpret_cast<VjpMemberDev*>(base + L.members);
  Tile* tiles = reinterpret_cast<Tile*>(base + L.tiles);
  const int grid_init = std::min((L.ntiles + kBlock - 1) / kBlock, 1024);
  vjp_single_plan<<<grid_init, kBlock, 0, st>>>(rec, dst, tiles, L.ntiles);
  return launch_ensemble_vjp(P, V, base, 1, L.ntiles, L.levelset,
                             align256(sizeof(uint32_t)), 0, st);
}

size_t spd_ensemble_vjp_plan_bytes(const spd_vjp_member_t* members, int nmembers) {
  if (!members || nmembers <= 0) return 0;
  return spd::plan_layout(members, nmembers, sizeof(spd::VjpMemberDev)).total;
}

int spd_ensemble_vjp_plan(const spd_class_t* classes, int nclasses,
                          const spd_vjp_member_t* members, int nmembers, void* plan_host,
                          void* plan_device, size_t plan_bytes, spd_plan_info_t* info) {
  using namespace spd;
  if (!classes || !members || !plan_host || !plan_device || !info) return SPD_ERR_NULL;
  if (nclasses <= 0 || nclasses > SPD_MAX_CLASSES || nmembers <= 0) return SPD_ERR_SHAPE;
  if (reinterpret_cast<uintptr_t>(plan_device) & 255u) return SPD_ERR_SCRATCH;
  const PlanLayout L = plan_layout(members, nmembers, sizeof(VjpMemberDev));
  if (plan_bytes < L.total) return SPD_ERR_SCRATCH;
  for (int i = 0; i < nmembers; ++i) {
    const spd_vjp_member_t& m = members[i];
    if (m.cls < 0 || m.cls >= nclasses) return SPD_ERR_SHAPE;
    spd_desc_t d = classes[m.cls].desc;
    d.ix = m.ix;
    d.il = m.il;
    const int rc = check_vjp_member(&d, &m.in, &m.ct, &m.grads);
    if (rc != SPD_OK) return rc;
  }
  char* h = static_cast<char*>(plan_host);
  memset(h, 0, L.total);
  VjpMemberDev* md = reinterpret_cast<VjpMemberDev*>(h + L.members);
  for (int i = 0; i < nmembers; ++i) {
    const spd_vjp_member_t& m = members[i];
    md[i].in = m.in;
    md[i].ct = m.ct;
    md[i].gr = m.grads;
    md[i].C = m.ix * m.il;
    md[i].il = m.il;
    md[i].kx = classes[m.cls].desc.kx;
    md[i].cls = m.cls;
  }
  const int t = plan_tiles(md, nmembers, L, static_cast<char*>(plan_device),
                           reinterpret_cast<Tile*>(h + L.tiles));
  info->nmembers = nmembers;
  info->ntiles = t;
  info->levelset_offset = L.levelset;
  info->levelset_bytes = align256((size_t)nmembers * sizeof(uint32_t));
  info->plan_bytes = L.total;
  return SPD_OK;
}

int spd_ensemble_vjp(const spd_class_t* classes, int nclasses, void* plan_device,
                     const spd_plan_info_t* info, int grid_blocks, void* stream) {
  using namespace spd;
  if (!classes || !plan_device || !info) return SPD_ERR_NULL;
  if (nclasses <= 0 || nclasses > SPD_MAX_CLASSES || info->ntiles <= 0) return SPD_ERR_SHAPE;
  ClassArgs P;
  VjpClassArgs V;
  for (int i = 0; i < nclasses; ++i) {
    P.cls[i].K = make_consts(&classes[i].desc, &classes[i].vgrid, &classes[i].params);
    P.cls[i].D = derive_constants(&classes[i].desc, &classes[i].vgrid, &classes[i].params);
    V.cls[i] = make_vjp_args(&classes[i].desc, &classes[i].vgrid, &classes[i].params);
  }
  // Default: one block per tile.  The blocks are short (one tile's columns each), so the SMs
  // turn over often and a higher-priority stream's kernels (a forward batch) get them within
  // one block's time; a persistent grid would hold every SM until the whole batch is done.
  return launch_ensemble_vjp(P, V, static_cast<char*>(plan_device), info->nmembers,
                             info->ntiles, info->levelset_offset, info->levelset_bytes,
                             grid_blocks, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
