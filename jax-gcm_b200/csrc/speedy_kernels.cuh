// speedy_kernels.cuh -- per-thread bodies shared by the plain and the ensemble kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "speedy_column_smem.cuh"

namespace spd {

constexpr int kBlock = 128;

template <int KX>
__device__ __forceinline__ void load_levels(const float* __restrict__ f, int C, int c, float v[KX]) {
#pragma unroll
  for (int k = 0; k < KX; ++k) v[k] = __ldg(f + (size_t)k * C + c);
}

// Level set of one block, OR-ed into the instance word once per block.
__device__ __forceinline__ void or_level_set(uint32_t bit, uint32_t* S) {
  __shared__ uint32_t warp_bits[kBlock / 32];  // one word per warp
  bit = __reduce_or_sync(0xffffffffu, bit);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_bits[warp] = bit;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t b = 0;
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) b |= warp_bits[w];
    const uint32_t have = *reinterpret_cast<volatile uint32_t*>(S);
    if ((have & b) != b) atomicOr(S, b);
  }
  __syncthreads();  // warp_bits may be rewritten by the caller's next tile
}

// Cloud-top level bit of column c from registers (the adjoint's pre-pass; the forward takes it
// from its first half).
template <int KX>
__device__ __forceinline__ uint32_t prepass_column(const Consts& K, const spd_inputs_t& in,
                                                   int c, int C) {
  float t[KX], q[KX], phi[KX];
  load_levels<KX>(in.temperature, C, c, t);
  load_levels<KX>(in.specific_humidity, C, c, q);
  load_levels<KX>(in.geopotential, C, c, phi);
  if (K.flags & SPD_FUSE_VERIFY) {
#pragma unroll
    for (int k = 0; k < KX; ++k) q[k] = (q[k] < 0.0f) ? 0.0f : q[k];
  }
  const float psa = __ldg(in.normalized_surface_pressure + c);
  const int icl = column_icltop<KX>(K, t, q, phi, psa);
  return 1u << min(max(icl, 0), KX - 1);
}

// Where the first launch leaves its results for the second, in the call's own output planes
// (the second launch rewrites every one of them): per level, the temperature and humidity
// tendency accumulators in out.temperature and out.specific_humidity and qsat in out.u_wind;
// per column, the scalars below in the first levels of out.v_wind (iptop and icltop as int
// bit patterns).  The two precipitation fields are final after the first half and go straight
// to their outputs.
enum { ST_CBMF, ST_CLOUDC, ST_CLSTR, ST_IPTOP, ST_ICLTOP, kStagedScalars };
static_assert(kStagedScalars <= 7, "the staged scalars fit the smallest level count");

// Loads the column's T, q (clamped at zero under SPD_FUSE_VERIFY) and phi into shared memory;
// returns the levels whose q was clamped.
template <int KX>
__device__ __forceinline__ uint32_t load_state(float* sm, const spd_inputs_t& in, bool verify,
                                               int c, int C) {
  float* tp = sm + (size_t)A_T * KX * kNT + threadIdx.x;
  float* qp = sm + (size_t)A_Q * KX * kNT + threadIdx.x;
  float* pp = sm + (size_t)A_PHI * KX * kNT + threadIdx.x;
  uint32_t neg = 0;
#pragma unroll 4
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    tp[k * kNT] = __ldg(in.temperature + i);
    float q = __ldg(in.specific_humidity + i);
    if (verify && q < 0.0f) {
      neg |= 1u << k;
      q = 0.0f;
    }
    qp[k * kNT] = q;
    pp[k * kNT] = __ldg(in.geopotential + i);
  }
  return neg;
}

// First half of column c (humidity through clouds), in registers: stages its results and
// returns the column's cloud-top level bit, 1 << clip(icltop, 0, kx-1).
template <int KX>
__device__ __forceinline__ uint32_t first_process(const ConstsD& CD, const spd_inputs_t& in,
                                                  const spd_outputs_t& out, int c, int C) {
  const bool verify = (CD.K.flags & SPD_FUSE_VERIFY) != 0;
  float t[KX], q[KX], phi[KX];
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    t[k] = __ldg(in.temperature + i);
    const float qk = __ldg(in.specific_humidity + i);
    q[k] = (verify && qk < 0.0f) ? 0.0f : qk;
    phi[k] = __ldg(in.geopotential + i);
  }
  SurfaceIn s;
  s.psa = __ldg(in.normalized_surface_pressure + c);
  s.fmask = __ldg(in.fmask + c);
  float qs[KX], dt[KX], dq[KX];
  ColScalars o;
  column_first<KX>(CD, t, q, phi, s, qs, dt, dq, o);
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    out.temperature[i] = dt[k];
    out.specific_humidity[i] = dq[k];
    out.u_wind[i] = qs[k];
  }
  out.v_wind[(size_t)ST_CBMF * C + c] = o.cbmf;
  out.v_wind[(size_t)ST_CLOUDC * C + c] = o.cloudc;
  out.v_wind[(size_t)ST_CLSTR * C + c] = o.clstr;
  out.v_wind[(size_t)ST_IPTOP * C + c] = __int_as_float(o.iptop);
  out.v_wind[(size_t)ST_ICLTOP * C + c] = __int_as_float(o.icltop);
  if (CD.K.flags & SPD_ACCUMULATE_DIAGNOSTICS) {
    out.precnv[c] = out.precnv[c] + o.precnv;
    out.precls[c] = out.precls[c] + o.precls;
  } else {
    __stcs(out.precnv + c, o.precnv);
    __stcs(out.precls + c, o.precls);
  }
  return 1u << min(max(o.icltop, 0), KX - 1);
}

// Horizontal part of the orographic correction of one column (orographic_correction.py:96-174):
// tcorh = gamlat phis0 and qcorh = refrh1 (qsat(tref) - qsat(tsfc, psfc)) with the land/sea
// surface temperature tsfc, tref = tsfc + tcorh and psfc = (tsfc / tref)^pexp.  The reference's
// get_qsat at sig <= 0 divides by the first element of a pressure field of ones
// (humidity.py:100-101), i.e. by 1 - 0.378 e.
__device__ __forceinline__ void orographic_horizontal(const Derived& D, float phis0, float fmask,
                                                      float stl, float sst, float& tcorh,
                                                      float& qcorh) {
  tcorh = D.gamlat * phis0;
  const float tsfc = fmask * stl + (1.0f - fmask) * sst;
  const float tref = tsfc + tcorh;
  const float psfc = powf(tsfc / tref, D.pexp);
  const float qref = qsat_of(tref, 1.0f, 1.0f);
  const float qsfc = qsat_of(tsfc, psfc, 1.0f);
  qcorh = 0.7f * (qref - qsfc);  // refrh1 (physical_constants.py:27)
}

// Second half of column c: reloads the state and the first half's stage, runs radiation,
// surface fluxes and vertical diffusion, applies verify_tendencies and stores every output.
// `sm` is the block's shared-memory arena laid out for KX levels.
template <int KX>
__device__ __forceinline__ void column_process(const ConstsD& CD, float* sm,
                                               const spd_inputs_t& in, const spd_outputs_t& out,
                                               const uint32_t* S,
                                               const ZonalRow* __restrict__ table, int c, int C,
                                               int il) {
  const Consts& K = CD.K;
  const bool verify = (K.flags & SPD_FUSE_VERIFY) != 0;
  const uint32_t neg = load_state<KX>(sm, in, verify, c, C);
  // Everything below reads the first launch's results (stage, level set, solar table).  When
  // this launch overlaps the first one's tail (programmatic dependent launch), wait here for
  // its completion; otherwise the first launch is complete already and this returns at once.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t Sw = *S;
  float* qsp = sm + (size_t)A_QSAT * KX * kNT + threadIdx.x;
  float* dtp = sm + (size_t)A_DT * KX * kNT + threadIdx.x;
  float* dqp = sm + (size_t)A_DQ * KX * kNT + threadIdx.x;
#pragma unroll 4
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    dtp[k * kNT] = __ldcs(out.temperature + i);
    dqp[k * kNT] = __ldcs(out.specific_humidity + i);
    qsp[k * kNT] = __ldcs(out.u_wind + i);
  }
  ColScalars o;
  o.cbmf = __ldcs(out.v_wind + (size_t)ST_CBMF * C + c);
  o.cloudc = __ldcs(out.v_wind + (size_t)ST_CLOUDC * C + c);
  o.clstr = __ldcs(out.v_wind + (size_t)ST_CLSTR * C + c);
  o.iptop = __float_as_int(__ldcs(out.v_wind + (size_t)ST_IPTOP * C + c));
  o.icltop = __float_as_int(__ldcs(out.v_wind + (size_t)ST_ICLTOP * C + c));
  SurfaceIn s;
  s.psa = __ldg(in.normalized_surface_pressure + c);
  s.u_low = __ldg(in.u_wind + (size_t)(KX - 1) * C + c);
  s.v_low = __ldg(in.v_wind + (size_t)(KX - 1) * C + c);
  s.sst = __ldg(in.sea_surface_temperature + c);
  s.stl = __ldg(in.stl_am + c);
  s.soilw = __ldg(in.soilw_am + c);
  s.snowc = __ldg(in.snowc_am + c);
  s.sice = __ldg(in.sice_am + c);
  s.alb0 = __ldg(in.alb0 + c);
  s.fmask = __ldg(in.fmask + c);
  s.orog = __ldg(in.orog + c);
  s.phis0 = __ldg(in.phis0 + c);
  const ZonalRow z = table[c % il];
  column_second<KX>(CD, sm, s, z, Sw, o);
  if (K.flags & SPD_OROGRAPHIC) {  // the last term (get_orographic_correction_tendencies)
    float tcorh, qcorh;
    orographic_horizontal(CD.D, s.phis0, s.fmask, s.stl, s.sst, tcorh, qcorh);
    const float dts = K.dt_seconds;
#pragma unroll 4
    for (int k = 0; k < KX; ++k) {
      dtp[k * kNT] = dtp[k * kNT] + (tcorh * CD.D.tcorv[k]) / dts;
      dqp[k * kNT] = dqp[k * kNT] + (qcorh * CD.D.qcorv[k]) / dts;
    }
  }
  const float* qp = sm + (size_t)A_Q * KX * kNT + threadIdx.x;
  // verify_tendencies (physics_interface.py:321-342) with the unclamped humidity
  if (verify) {
    const float dt = K.dt_seconds;
#pragma unroll 1
    for (int k = 0; k < KX; ++k) {
      const float qr = (neg >> k & 1u) ? __ldg(in.specific_humidity + (size_t)k * C + c)
                                       : qp[k * kNT];
      const float dq = dqp[k * kNT];
      dqp[k * kNT] = (qr + dt * dq >= 0.0f) ? dq : -qr / dt;
    }
  }
  const float qs = K.q_tend_scale;
#pragma unroll 4
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    __stcs(out.u_wind + i, k == KX - 1 ? o.du_low : 0.0f);
    __stcs(out.v_wind + i, k == KX - 1 ? o.dv_low : 0.0f);
    __stcs(out.temperature + i, dtp[k * kNT]);
    const float dq = dqp[k * kNT];
    __stcs(out.specific_humidity + i, qs != 1.0f ? dq * qs : dq);
  }
  // diagnostics: stored, or added to the caller's sums under SPD_ACCUMULATE_DIAGNOSTICS
  const bool acc = (K.flags & SPD_ACCUMULATE_DIAGNOSTICS) != 0;
  auto put = [&](float* f, float x) {
    if (f) f[c] = acc ? f[c] + x : x;
  };
  put(out.cbmf, o.cbmf);
  put(out.cloudc, o.cloudc);
  put(out.cloudstr, o.clstr);
  put(out.rsds, o.rsds);
  put(out.rsns, o.rsns);
  put(out.ftop_sw, o.ftop_sw);
  put(out.rlds, o.rlds);
  put(out.rlns, o.rlns);
  put(out.ftop_lw, o.ftop_lw);
  put(out.tsfc, o.tsfc);
  put(out.tskin, o.tskin);
  put(out.shf, o.shf);
  put(out.evap, o.evap);
  if (out.iptop) out.iptop[c] = o.iptop;
  if (out.icltop) out.icltop[c] = o.icltop;
}

}  // namespace spd
