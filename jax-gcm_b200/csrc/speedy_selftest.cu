// speedy_selftest.cu -- spd_selftest_packed: the forward's packed float32 pieces
// (speedy_column_smem.cuh: lw_step, radset_w, th_pair, bb_pair, sw_band1, sw_band2, sw_scale)
// against the scalar expressions they pair, bit for bit, on seeded inputs.  Compiled with the
// forward's flags (no contraction, approximate division, subnormal flush), so a compiler that
// fused a packed product into a sum, or rounded a lane differently, shows up as a mismatch
// here before it shows up as a parity drift.
#include <cuda_runtime.h>
#include <stdint.h>

#include "speedy_column_smem.cuh"

namespace spd {
namespace {

__device__ __forceinline__ uint32_t mix(uint32_t x) {  // a 32-bit integer hash (xorshift-multiply)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Uniform in [lo, hi); every 61st draw an edge value: zero, a subnormal, or the bound itself.
__device__ __forceinline__ float draw(uint32_t& s, float lo, float hi) {
  s = mix(s + 0x9e3779b9u);
  if (s % 61u == 0u) {
    const uint32_t e = (s >> 8) % 3u;
    return e == 0u ? 0.0f : (e == 1u ? 1.0e-39f : lo);
  }
  return lo + (hi - lo) * ((s >> 8) * (1.0f / 16777216.0f));
}

__device__ __forceinline__ bool differ(float a, float b) {
  return __float_as_uint(a) != __float_as_uint(b);
}

enum { M_LW_DOWN, M_LW_UP, M_RADSET, M_TH, M_BB, M_SW1, M_SW2, M_SCALE, kNumChecks };

__global__ void selftest_packed(int n, uint32_t seed, unsigned int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t s = mix(seed ^ mix((uint32_t)i));
  unsigned int local[kNumChecks] = {};
  // longwave recurrence, one band pair, both directions
  {
    const float2 tau = pk(draw(s, 0.0f, 1.0f), draw(s, 0.0f, 1.0f));
    const float2 fl = pk(draw(s, 0.0f, 500.0f), draw(s, 0.0f, 500.0f));
    const float2 fb = pk(draw(s, 0.0f, 1.0f), draw(s, 0.0f, 1.0f));
    const float s0 = draw(s, 0.0f, 500.0f), s1 = draw(s, 0.0f, 50.0f);
    const float2 dn = lw_step<true>(tau, fl, fb, s0, s1);
    const float2 up = lw_step<false>(tau, fl, fb, s0, s1);
    const float e0 = 1.0f - tau.x, e1 = 1.0f - tau.y;
    local[M_LW_DOWN] += differ(dn.x, tau.x * fl.x + e0 * (fb.x * (s0 + e0 * s1)));
    local[M_LW_DOWN] += differ(dn.y, tau.y * fl.y + e1 * (fb.y * (s0 + e1 * s1)));
    local[M_LW_UP] += differ(up.x, tau.x * fl.x + e0 * (fb.x * (s0 - e0 * s1)));
    local[M_LW_UP] += differ(up.y, tau.y * fl.y + e1 * (fb.y * (s0 - e1 * s1)));
  }
  // band energy fractions (longwave_radiation.py:204-226)
  {
    const float temp = draw(s, 150.0f, 350.0f), w = draw(s, 0.0f, 1.0f);
    float2 fb01, fb23;
    radset_w(temp, w, fb01, fb23);
    const float j = fminf(fmaxf(temp, 200.0f), 320.0f);
    const float f1 = 0.148f - 3.0e-6f * sq(j - 247.0f);
    const float f2 = 0.356f - 5.2e-6f * sq(j - 282.0f);
    const float f3 = 0.314f + 1.0e-5f * sq(j - 315.0f);
    const float f0 = 1.0f - (((0.0f + f1) + f2) + f3);
    local[M_RADSET] += differ(fb01.x, w * f0) + differ(fb01.y, w * f1) +
                       differ(fb23.x, w * f2) + differ(fb23.y, w * f3);
  }
  // half-level temperatures and blackbody terms
  {
    const float tm = draw(s, 180.0f, 320.0f), t = draw(s, 180.0f, 320.0f),
                tp = draw(s, 180.0f, 320.0f);
    const float wk = draw(s, 0.0f, 1.0f), wm = draw(s, 0.0f, 1.0f);
    const float2 th = th_pair(tm, t, tp, wk, wm);
    local[M_TH] += differ(th.x, t + wk * (tp - t)) + differ(th.y, tm + wm * (t - tm));
    const float2 bb = bb_pair(t);
    const float st3 = kSbc * (t * t * t);
    local[M_BB] += differ(bb.x, st3 * t) + differ(bb.y, 4.0f * st3);
  }
  // shortwave pieces
  {
    const float prev = draw(s, 0.0f, 1400.0f), r = draw(s, 0.0f, 0.5f), t0 = draw(s, 0.0f, 1.0f);
    const float2 fd = sw_band1(prev, r, t0);
    local[M_SW1] += differ(fd.x, prev * t0 * (1.0f - r)) +
                    differ(fd.y, prev * (1.0f - r) * (1.0f - t0));
    const float prev2 = draw(s, 0.0f, 80.0f), tau1 = draw(s, 0.0f, 1.0f);
    const float2 f2 = sw_band2(prev2, tau1);
    local[M_SW2] += differ(f2.x, prev2 * tau1) + differ(f2.y, prev2 * (1.0f - tau1));
    const float a = draw(s, 0.0f, 100.0f), b = draw(s, 0.0f, 100.0f);
    const float g = draw(s, 0.0f, 1.0e-3f), rps = draw(s, 0.9f, 1.1f);
    const float2 sc = sw_scale(a, b, g, rps);
    local[M_SCALE] += differ(sc.x, a * g * rps) + differ(sc.y, b * g * rps);
  }
#pragma unroll
  for (int c = 0; c < kNumChecks; ++c)
    if (local[c]) atomicAdd(bad + c, local[c]);
}

}  // namespace
}  // namespace spd

extern "C" int spd_selftest_packed(int n, uint32_t seed, unsigned int* mismatches) {
  using namespace spd;
  if (!mismatches) return SPD_ERR_NULL;
  if (n <= 0) return SPD_ERR_SHAPE;
  unsigned int* d = nullptr;
  if (cudaMalloc(&d, kNumChecks * sizeof(unsigned int)) != cudaSuccess) return SPD_ERR_CUDA;
  int rc = SPD_OK;
  if (cudaMemset(d, 0, kNumChecks * sizeof(unsigned int)) != cudaSuccess) rc = SPD_ERR_CUDA;
  if (rc == SPD_OK) {
    selftest_packed<<<(n + 255) / 256, 256>>>(n, seed, d);
    if (cudaGetLastError() != cudaSuccess) rc = SPD_ERR_CUDA;
  }
  if (rc == SPD_OK && cudaMemcpy(mismatches, d, kNumChecks * sizeof(unsigned int),
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = SPD_ERR_CUDA;
  cudaFree(d);
  return rc;
}
