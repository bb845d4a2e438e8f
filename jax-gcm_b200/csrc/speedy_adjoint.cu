// speedy_adjoint.cu -- the adjoint of the plain forward (spd_vjp).
//
// Launch 1 is the forward's cloud-top pre-pass (the instance level set S and the per-latitude
// solar table: neither carries a derivative).  Launch 2 runs one thread per column: the
// hand-written reverse pass of speedy_vjp.h recomputes the column's forward and walks its terms
// backwards, writing the state gradients.  The 12 parameter gradients are summed per thread,
// then per block, then with one atomicAdd per block and parameter.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "speedy_kernels.cuh"
#include "speedy_vjp.h"

namespace spd {

int check_instance(const spd_desc_t* d, const spd_inputs_t* in, const spd_outputs_t* out);
Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p);

constexpr size_t kAdjHeader = 256;
constexpr int kAdjBlock = 128;

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

inline size_t vjp_scratch(const spd_desc_t* d) {
  return kAdjHeader + align256((size_t)d->il * sizeof(ZonalRow));
}

struct VjpArgs {
  spd_vgrid_t vg;
  spd_params_t p;
  uint32_t flags;
  int model_step, C, il;
  float ablco2, dt_seconds, q_tend_scale;
};

template <int KX>
__global__ void __launch_bounds__(kAdjBlock)
    adjoint_kernel(const __grid_constant__ VjpArgs A, const spd_inputs_t in,
                   const spd_cotangents_t ct, const spd_grads_t gr,
                   const uint32_t* __restrict__ S, const ZonalRow* __restrict__ table) {
  const int C = A.C;
  const spdvjp::Ctx x{&A.vg, &A.p, A.flags, A.model_step, __ldg(S)};
  spdgen::DiffParams<float> g;
  g.psmin = A.p.psmin; g.trcnv = A.p.trcnv; g.rhil = A.p.rhil; g.rhbl = A.p.rhbl;
  g.entmax = A.p.entmax; g.smf = A.p.smf; g.trlsc = A.p.trlsc; g.rhlsc = A.p.rhlsc;
  g.drhlsc = A.p.drhlsc; g.rhblsc = A.p.rhblsc; g.albcl = A.p.albcl; g.albcls = A.p.albcls;
  float pacc[SPD_NUM_DIFF_PARAMS];
#pragma unroll
  for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) pacc[j] = 0.0f;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    spdgen::ColumnIn<float, float> xi;
    float ct_t[KX], ct_q[KX];
#pragma unroll 1
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
    const ZonalRow z = table[c % A.il];
    xi.fsol = z.fsol; xi.ozupp = z.ozupp; xi.ozone = z.ozone; xi.zenit = z.zenit;
    xi.stratz = z.stratz; xi.sqrt_coa = z.sqrt_coa;
    spdvjp::Bar<KX, float> b;
    spdvjp::column_vjp<KX, float>(x, g, A.ablco2, A.dt_seconds, A.q_tend_scale, xi, ct_t, ct_q,
                                  __ldg(ct.u_wind + lo), __ldg(ct.v_wind + lo), b);
#pragma unroll 1
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
  // parameter gradients: warp, then block, then one atomic per block and parameter
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
    atomicAdd(gr.params + threadIdx.x, v);
  }
}

template <int KX>
static int launch_vjp(const VjpArgs& A, const Consts& K, const spd_inputs_t& in,
                      const spd_cotangents_t& ct, const spd_grads_t& gr, char* scratch,
                      cudaStream_t st) {
  uint32_t* S = reinterpret_cast<uint32_t*>(scratch);
  ZonalRow* table = reinterpret_cast<ZonalRow*>(scratch + kAdjHeader);
  const int grid_a = (std::max(K.C, K.il) + kBlock - 1) / kBlock;
  cloudtop_prepass<KX><<<grid_a, kBlock, 0, st>>>(K, in, S, table);
  const int grid = (A.C + kAdjBlock - 1) / kAdjBlock;
  adjoint_kernel<KX><<<grid, kAdjBlock, 0, st>>>(A, in, ct, gr, S, table);
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}

}  // namespace spd

extern "C" {

size_t spd_vjp_scratch_bytes(const spd_desc_t* desc) {
  if (!desc || desc->ix <= 0 || desc->il <= 0) return 0;
  return spd::vjp_scratch(desc);
}

int spd_vjp(const spd_desc_t* desc, const spd_vgrid_t* vgrid, const spd_params_t* params,
            const spd_inputs_t* in, const spd_cotangents_t* ct, const spd_grads_t* grads,
            void* scratch, size_t scratch_bytes, void* stream) {
  using namespace spd;
  if (!desc || !vgrid || !params || !in || !ct || !grads) return SPD_ERR_NULL;
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
  if (!scratch || (reinterpret_cast<uintptr_t>(scratch) & 255u) ||
      scratch_bytes < vjp_scratch(desc))
    return SPD_ERR_SCRATCH;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Consts K = make_consts(desc, vgrid, params);
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
  char* sc = static_cast<char*>(scratch);
  if (cudaMemsetAsync(sc, 0, kAdjHeader, st) != cudaSuccess) return SPD_ERR_CUDA;
  if (cudaMemsetAsync(grads->params, 0, SPD_NUM_DIFF_PARAMS * sizeof(float), st) != cudaSuccess)
    return SPD_ERR_CUDA;
  switch (desc->kx) {
    case 7: return launch_vjp<7>(A, K, *in, *ct, *grads, sc, st);
    case 8: return launch_vjp<8>(A, K, *in, *ct, *grads, sc, st);
    case 16: return launch_vjp<16>(A, K, *in, *ct, *grads, sc, st);
    default: return SPD_ERR_KX;
  }
}

}  // extern "C"
