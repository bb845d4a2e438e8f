// speedy_adjoint.cu -- recompute-in-column adjoint of the plain forward (spd_vjp).
//
// Launch 1 is the forward's cloud-top pre-pass (the instance level set S and the per-latitude
// solar table: neither carries a derivative).  Launch 2 gives every thread a slice of the tape
// scratch; per column it records the column's forward on the tape (speedy_generic.h with
// R = Adj<float>), seeds the output adjoints with the cotangents, sweeps the tape once and
// writes the input gradients.  The 12 parameter gradients are summed per thread, then per block,
// then with one atomicAdd per block and parameter.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "speedy_generic.h"
#include "speedy_kernels.cuh"

namespace spd {

int check_instance(const spd_desc_t* d, const spd_inputs_t* in, const spd_outputs_t* out);
Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p);

constexpr size_t kAdjHeader = 256;

inline int tape_cap(int kx) { return 320 * kx + 512; }

inline int vjp_threads(int C) {
  const int t = ((C + kBlock - 1) / kBlock) * kBlock;
  return std::min(t, SPD_VJP_MAX_THREADS);
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct VjpLayout {
  size_t table, ia, ib, pa, pb, adj, total;
  int cap, nthreads;
};

inline VjpLayout vjp_layout(const spd_desc_t* d) {
  VjpLayout L;
  const int C = d->ix * d->il;
  L.cap = tape_cap(d->kx);
  L.nthreads = vjp_threads(C);
  const size_t per = (size_t)L.cap * L.nthreads * 4;
  L.table = kAdjHeader;
  L.ia = L.table + align256((size_t)d->il * sizeof(ZonalRow));
  L.ib = L.ia + align256(per);
  L.pa = L.ib + align256(per);
  L.pb = L.pa + align256(per);
  L.adj = L.pb + align256(per);
  L.total = L.adj + align256(per);
  return L;
}

struct VjpArgs {
  spd_vgrid_t vg;
  spd_params_t p;
  uint32_t flags;
  int model_step, C, il, cap;
  float ablco2, dt_seconds, q_tend_scale;
};

template <int KX>
__global__ void __launch_bounds__(kBlock) adjoint_kernel(const VjpArgs A, const spd_inputs_t in,
                                                         const spd_cotangents_t ct,
                                                         const spd_grads_t gr,
                                                         const uint32_t* __restrict__ S,
                                                         const ZonalRow* __restrict__ table,
                                                         int32_t* ia, int32_t* ib, float* pa,
                                                         float* pb, float* adj,
                                                         uint32_t* status) {
  using spdad::Adj;
  typedef Adj<float> AF;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthr = gridDim.x * blockDim.x;
  spdad::TapeT<float> tp{ia + gtid, ib + gtid, pa + gtid, pb + gtid, adj + gtid,
                         (size_t)nthr, 0, A.cap, 0};
  const int C = A.C;
  const uint32_t Sw = __ldg(S);
  const bool verify = (A.flags & SPD_FUSE_VERIFY) != 0;
  float pacc[SPD_NUM_DIFF_PARAMS];
#pragma unroll
  for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) pacc[j] = 0.0f;
  for (int c = gtid; c < C; c += nthr) {
    tp.n = 0;
    auto leaf = [&](float v) { return AF(v, tp.leaf(), &tp); };
    spdgen::DiffParams<AF> g;
    g.psmin = leaf(A.p.psmin); g.trcnv = leaf(A.p.trcnv); g.rhil = leaf(A.p.rhil);
    g.rhbl = leaf(A.p.rhbl); g.entmax = leaf(A.p.entmax); g.smf = leaf(A.p.smf);
    g.trlsc = leaf(A.p.trlsc); g.rhlsc = leaf(A.p.rhlsc); g.drhlsc = leaf(A.p.drhlsc);
    g.rhblsc = leaf(A.p.rhblsc); g.albcl = leaf(A.p.albcl); g.albcls = leaf(A.p.albcls);
    spdgen::ColumnIn<AF, float> x;
    AF qraw[KX];
    for (int k = 0; k < KX; ++k) {
      const size_t i = (size_t)k * C + c;
      x.t[k] = leaf(__ldg(in.temperature + i));
      qraw[k] = leaf(__ldg(in.specific_humidity + i));
      // verify_state (physics_interface.py:316): where(q < 0, 0, q)
      x.q[k] = (verify && qraw[k].v < 0.0f) ? AF(0.0f) : qraw[k];
      x.phi[k] = leaf(__ldg(in.geopotential + i));
    }
    x.psa = leaf(__ldg(in.normalized_surface_pressure + c));
    x.u_low = leaf(__ldg(in.u_wind + (size_t)(KX - 1) * C + c));
    x.v_low = leaf(__ldg(in.v_wind + (size_t)(KX - 1) * C + c));
    x.sst = __ldg(in.sea_surface_temperature + c);
    x.stl = __ldg(in.stl_am + c);
    x.soilw = __ldg(in.soilw_am + c);
    x.snowc = __ldg(in.snowc_am + c);
    x.sice = __ldg(in.sice_am + c);
    x.alb0 = __ldg(in.alb0 + c);
    x.fmask = __ldg(in.fmask + c);
    x.orog = __ldg(in.orog + c);
    x.phis0 = __ldg(in.phis0 + c);
    const ZonalRow z = table[c % A.il];
    x.fsol = z.fsol; x.ozupp = z.ozupp; x.ozone = z.ozone; x.zenit = z.zenit;
    x.stratz = z.stratz; x.sqrt_coa = z.sqrt_coa;
    spdgen::ColumnOut<AF> o;
    spdgen::column_generic<KX, AF, float>(A.vg, A.p, g, A.flags, A.model_step, A.ablco2, Sw, x,
                                          o);
    for (int k = 0; k < KX; ++k) {
      AF dq = o.dq[k];
      if (verify) {  // verify_tendencies (physics_interface.py:334-340)
        dq = (qraw[k].v + A.dt_seconds * dq.v >= 0.0f) ? dq : -qraw[k] / A.dt_seconds;
      }
      if (A.q_tend_scale != 1.0f) dq = dq * A.q_tend_scale;
      const size_t i = (size_t)k * C + c;
      tp.seed(o.dt[k].i, __ldg(ct.temperature + i));
      tp.seed(dq.i, __ldg(ct.specific_humidity + i));
    }
    tp.seed(o.du_low.i, __ldg(ct.u_wind + (size_t)(KX - 1) * C + c));
    tp.seed(o.dv_low.i, __ldg(ct.v_wind + (size_t)(KX - 1) * C + c));
    tp.reverse();
    for (int k = 0; k < KX; ++k) {
      const size_t i = (size_t)k * C + c;
      gr.temperature[i] = tp.grad(x.t[k].i);
      gr.specific_humidity[i] = tp.grad(qraw[k].i);
      gr.geopotential[i] = tp.grad(x.phi[k].i);
      gr.u_wind[i] = (k == KX - 1) ? tp.grad(x.u_low.i) : 0.0f;
      gr.v_wind[i] = (k == KX - 1) ? tp.grad(x.v_low.i) : 0.0f;
    }
    gr.normalized_surface_pressure[c] = tp.grad(x.psa.i);
    const int pidx[SPD_NUM_DIFF_PARAMS] = {g.psmin.i, g.trcnv.i, g.rhil.i,   g.rhbl.i,
                                           g.entmax.i, g.smf.i,   g.trlsc.i,  g.rhlsc.i,
                                           g.drhlsc.i, g.rhblsc.i, g.albcl.i, g.albcls.i};
#pragma unroll
    for (int j = 0; j < SPD_NUM_DIFF_PARAMS; ++j) pacc[j] += tp.grad(pidx[j]);
    if (tp.overflow) atomicOr(status, 1u);
  }
  // parameter gradients: warp, then block, then one atomic per block and parameter
  __shared__ float red[kBlock / 32][SPD_NUM_DIFF_PARAMS];
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
    for (int w = 0; w < kBlock / 32; ++w) v += red[w][threadIdx.x];
    atomicAdd(gr.params + threadIdx.x, v);
  }
}

template <int KX>
static int launch_vjp(const VjpArgs& A, const Consts& K, const spd_inputs_t& in,
                      const spd_cotangents_t& ct, const spd_grads_t& gr, char* scratch,
                      const VjpLayout& L, cudaStream_t st) {
  uint32_t* S = reinterpret_cast<uint32_t*>(scratch);
  uint32_t* status = S + 1;
  ZonalRow* table = reinterpret_cast<ZonalRow*>(scratch + L.table);
  const int grid_a = (std::max(K.C, K.il) + kBlock - 1) / kBlock;
  cloudtop_prepass<KX><<<grid_a, kBlock, 0, st>>>(K, in, S, table);
  adjoint_kernel<KX><<<L.nthreads / kBlock, kBlock, 0, st>>>(
      A, in, ct, gr, S, table, reinterpret_cast<int32_t*>(scratch + L.ia),
      reinterpret_cast<int32_t*>(scratch + L.ib), reinterpret_cast<float*>(scratch + L.pa),
      reinterpret_cast<float*>(scratch + L.pb), reinterpret_cast<float*>(scratch + L.adj),
      status);
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}

}  // namespace spd

extern "C" {

size_t spd_vjp_scratch_bytes(const spd_desc_t* desc) {
  if (!desc || desc->ix <= 0 || desc->il <= 0) return 0;
  return spd::vjp_layout(desc).total;
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
  const VjpLayout L = vjp_layout(desc);
  if (!scratch || (reinterpret_cast<uintptr_t>(scratch) & 255u) || scratch_bytes < L.total)
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
  A.cap = L.cap;
  A.ablco2 = D.ablco2;
  A.dt_seconds = desc->dt_seconds;
  A.q_tend_scale = desc->q_tend_scale;
  char* sc = static_cast<char*>(scratch);
  if (cudaMemsetAsync(sc, 0, kAdjHeader, st) != cudaSuccess) return SPD_ERR_CUDA;
  if (cudaMemsetAsync(grads->params, 0, SPD_NUM_DIFF_PARAMS * sizeof(float), st) != cudaSuccess)
    return SPD_ERR_CUDA;
  switch (desc->kx) {
    case 7: return launch_vjp<7>(A, K, *in, *ct, *grads, sc, L, st);
    case 8: return launch_vjp<8>(A, K, *in, *ct, *grads, sc, L, st);
    case 16: return launch_vjp<16>(A, K, *in, *ct, *grads, sc, L, st);
    default: return SPD_ERR_KX;
  }
}

}  // extern "C"
