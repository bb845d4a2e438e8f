// held_suarez.cu -- spd_held_suarez: the Held-Suarez forcing
// (jcm/physics/held_suarez/held_suarez_physics.py), the reference's second physics package.
//
// Every element is independent: relaxation of T towards the radiative-equilibrium temperature
// and Rayleigh drag on u and v, no humidity tendency.  Per level and column the call moves 28
// bytes (u, v, T read; du, dv, dT, dq written) plus psa once per column, against a few dozen
// instructions, so it is bound by HBM.  One thread takes four consecutive columns at two
// levels: 128-bit loads and stores (float4) of the level planes, psa and the latitude terms
// loaded once per item; one item per thread.  Shapes whose planes are not 16-byte aligned (or
// whose column count is not a multiple of 4) take a path with one column per thread, walking its
// levels, at most eight 256-thread blocks per SM and grid-stride beyond.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "speedy_b200.h"

namespace {

struct HsConsts {
  int kx, C, il;
  float ka, ksa;  // ka and ks - ka
  float min_t, max_t, dt_y, dthz, kappa;
  float sigma[SPD_MAX_KX];   // level centres
  float cutoff[SPD_MAX_KX];  // max(0, (sigma - sigma_b) / (1 - sigma_b))
  float kv[SPD_MAX_KX];      // kf * cutoff
};

// Temperature tendency of one element (held_suarez_physics.py:53-62, :70-74, :92-93).
// p^kappa is formed as exp(kappa log p) from the log the equilibrium temperature needs anyway
// (a general power costs several times more; for p = sigma psa <= ~1.1 the two agree to a
// few float32 ulp).
__device__ __forceinline__ float hs_dt(const HsConsts& H, int k, float t, float psa, float s2,
                                       float c2, float c4) {
  const float p = H.sigma[k] * psa;  // p_over_p0
  const float lp = logf(p);
  const float teq =
      fmaxf(H.min_t, expf(H.kappa * lp) * ((H.max_t - H.dt_y * s2) - H.dthz * lp * c2));
  const float kt = H.ka + H.ksa * (H.cutoff[k] * c4);
  return -kt * (t - teq);
}

// Work items of kHsChunk levels of one group of four columns, level chunk outermost: a call is
// many waves of short blocks instead of 1.35 waves of long ones (the partial last wave of the
// column-group form left most SMs idle for a third of the call), and each chunk re-reads only
// psa and the latitude rows, which stay in L2 between chunks.  Measured at T425 with 16
// levels: all 16 levels per item 0.068 ms (83 % of the measured copy bandwidth); 8 or 4 levels
// 0.065 ms; 2 levels 0.061 ms (93 %); 1 level 0.065 ms.
constexpr int kHsChunk = 2;

__global__ void __launch_bounds__(256) hs_vec4(const HsConsts H, const float* __restrict__ lat,
                                               const float4* __restrict__ u,
                                               const float4* __restrict__ v,
                                               const float4* __restrict__ t,
                                               const float4* __restrict__ psa,
                                               float4* __restrict__ du, float4* __restrict__ dv,
                                               float4* __restrict__ dt, float4* __restrict__ dq) {
  const int C4 = H.C / 4;
  const int nchunks = (H.kx + kHsChunk - 1) / kHsChunk;
  const int64_t nitems = (int64_t)C4 * nchunks;
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < nitems;
       it += (int64_t)gridDim.x * blockDim.x) {
    const int kc = (int)(it / C4);
    const int g = (int)(it - (int64_t)kc * C4);
    const float4 ps = __ldg(psa + g);
    const int j0 = (4 * g) % H.il;
    float s2[4], c2[4], c4[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = (j0 + i) % H.il;
      s2[i] = __ldg(lat + j);
      c2[i] = __ldg(lat + H.il + j);
      c4[i] = __ldg(lat + 2 * H.il + j);
    }
    const int k0 = kc * kHsChunk;
#pragma unroll
    for (int dk = 0; dk < kHsChunk; ++dk) {
      const int k = k0 + dk;
      if (k >= H.kx) break;
      const size_t e = (size_t)k * C4 + g;
      const float4 uu = __ldcs(u + e), vv = __ldcs(v + e), tt = __ldcs(t + e);
      const float kv = H.kv[k];
      __stcs(du + e, make_float4(-kv * uu.x, -kv * uu.y, -kv * uu.z, -kv * uu.w));
      __stcs(dv + e, make_float4(-kv * vv.x, -kv * vv.y, -kv * vv.z, -kv * vv.w));
      __stcs(dt + e, make_float4(hs_dt(H, k, tt.x, ps.x, s2[0], c2[0], c4[0]),
                                 hs_dt(H, k, tt.y, ps.y, s2[1], c2[1], c4[1]),
                                 hs_dt(H, k, tt.z, ps.z, s2[2], c2[2], c4[2]),
                                 hs_dt(H, k, tt.w, ps.w, s2[3], c2[3], c4[3])));
      __stcs(dq + e, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    }
  }
}

__global__ void __launch_bounds__(256) hs_scalar(const HsConsts H, const float* __restrict__ lat,
                                                 const float* __restrict__ u,
                                                 const float* __restrict__ v,
                                                 const float* __restrict__ t,
                                                 const float* __restrict__ psa,
                                                 float* __restrict__ du, float* __restrict__ dv,
                                                 float* __restrict__ dt, float* __restrict__ dq) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < H.C; c += gridDim.x * blockDim.x) {
    const float ps = __ldg(psa + c);
    const int j = c % H.il;
    const float s2 = __ldg(lat + j), c2 = __ldg(lat + H.il + j), c4 = __ldg(lat + 2 * H.il + j);
#pragma unroll 4
    for (int k = 0; k < H.kx; ++k) {
      const size_t e = (size_t)k * H.C + c;
      const float kv = H.kv[k];
      du[e] = -kv * __ldg(u + e);
      dv[e] = -kv * __ldg(v + e);
      dt[e] = hs_dt(H, k, __ldg(t + e), ps, s2, c2, c4);
      dq[e] = 0.0f;
    }
  }
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// True when [a, a + na) and [b, b + nb) (floats) overlap.
bool overlap(const float* a, size_t na, const float* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb * sizeof(float) && y < x + na * sizeof(float);
}

}  // namespace

namespace spd {
int preload_held_suarez() {
  cudaFuncAttributes a;
  bool ok = cudaFuncGetAttributes(&a, hs_vec4) == cudaSuccess;
  ok &= cudaFuncGetAttributes(&a, hs_scalar) == cudaSuccess;
  return ok ? SPD_OK : SPD_ERR_CUDA;
}
}  // namespace spd

extern "C" int spd_held_suarez(const spd_hs_desc_t* d, const float* lat_tab, const float* u,
                               const float* v, const float* t, const float* psa, float* du,
                               float* dv, float* dt, float* dq, void* stream) {
  if (!d || !lat_tab || !u || !v || !t || !psa || !du || !dv || !dt || !dq) return SPD_ERR_NULL;
  if (d->kx < 1 || d->kx > SPD_MAX_KX) return SPD_ERR_KX;
  if (d->ix <= 0 || d->il <= 0 || (int64_t)d->ix * d->il > (1 << 30)) return SPD_ERR_SHAPE;
  {
    const size_t C = (size_t)d->ix * d->il, L = (size_t)d->kx * C;
    const float* ins[] = {u, v, t};
    float* outs[] = {du, dv, dt, dq};
    for (int i = 0; i < 4; ++i) {
      for (const float* p : ins)
        if (overlap(outs[i], L, p, L)) return SPD_ERR_ALIAS;
      if (overlap(outs[i], L, psa, C)) return SPD_ERR_ALIAS;
      for (int j = 0; j < i; ++j)
        if (overlap(outs[i], L, outs[j], L)) return SPD_ERR_ALIAS;
    }
  }
  HsConsts H;
  H.kx = d->kx;
  H.C = d->ix * d->il;
  H.il = d->il;
  H.ka = d->ka;
  H.ksa = d->ks - d->ka;
  H.min_t = d->min_t;
  H.max_t = d->max_t;
  H.dt_y = d->dt_y;
  H.dthz = d->dthz;
  H.kappa = d->kappa;
  for (int k = 0; k < SPD_MAX_KX; ++k) {
    const float s = k < d->kx ? d->sigma[k] : 0.0f;
    H.sigma[k] = s;
    H.cutoff[k] = std::max(0.0f, (s - d->sigma_b) / (1.0f - d->sigma_b));  // :65-67, :71
    H.kv[k] = d->kf * H.cutoff[k];
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return SPD_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const void* planes[] = {u, v, t, psa, du, dv, dt, dq};
  bool vec = (H.C % 4) == 0;
  for (const void* p : planes) vec = vec && aligned16(p);
  const int threads = 256;
  if (vec) {
    // one work item (four columns, up to kHsChunk levels) per thread
    const int64_t items = (int64_t)(H.C / 4) * ((H.kx + kHsChunk - 1) / kHsChunk);
    const int grid = (int)std::min<int64_t>((items + threads - 1) / threads, (int64_t)1 << 30);
    hs_vec4<<<grid, threads, 0, st>>>(
        H, lat_tab, reinterpret_cast<const float4*>(u), reinterpret_cast<const float4*>(v),
        reinterpret_cast<const float4*>(t), reinterpret_cast<const float4*>(psa),
        reinterpret_cast<float4*>(du), reinterpret_cast<float4*>(dv),
        reinterpret_cast<float4*>(dt), reinterpret_cast<float4*>(dq));
  } else {
    // grid: enough blocks to cover the columns, at most 8 per SM (grid-stride beyond)
    const int grid = (int)std::min<int64_t>((H.C + threads - 1) / threads, (int64_t)sms * 8);
    hs_scalar<<<grid, threads, 0, st>>>(H, lat_tab, u, v, t, psa, du, dv, dt, dq);
  }
  return cudaGetLastError() == cudaSuccess ? SPD_OK : SPD_ERR_CUDA;
}
