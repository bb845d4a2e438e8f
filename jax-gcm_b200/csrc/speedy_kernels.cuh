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

// The fused launch's form of or_level_set: the OR of a warp's bits, added by one lane, with no
// block barrier (the fused launch's warps run their columns at very different speeds, and a
// barrier per tile would hold the fast ones).  Every lane of the warp must call it.
__device__ __forceinline__ void or_level_set_warp(uint32_t bit, uint32_t* S) {
  bit = __reduce_or_sync(0xffffffffu, bit);
  if ((threadIdx.x & 31) == 0) {
    const uint32_t have = *reinterpret_cast<volatile uint32_t*>(S);
    if ((have & bit) != bit) atomicOr(S, bit);
  }
}

// Cloud-top level bit of column c from registers (the adjoint's pre-pass; the forward forms it
// from its own first half, column_first).
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

// Cloud-top level bit of column c, 1 << clip(icltop, 0, kx-1), from the forward's own first
// half in its top-only form (the level-set launch).
template <int KX>
__device__ __forceinline__ uint32_t levelset_bit(const ConstsD& CD, const spd_inputs_t& in,
                                                 int c, int C) {
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
  s.fmask = 0.0f;
  float qs[KX], dt[KX], dq[KX];
  ColScalars o;
  column_first<KX, true>(CD, t, q, phi, s, qs, dt, dq, o);
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

// The end of column c, shared by the forward's kernels: the orographic correction (the last
// term, when on), verify_tendencies, the tendency stores and the diagnostics.  The level arrays
// T, Q (clamped by verify_state where `neg` has a bit), the accumulated tendencies DT and DQ are
// in the block's shared-memory arena; o holds the column's scalar results.
template <int KX>
__device__ __forceinline__ void column_outputs(const ConstsD& CD, float* sm,
                                               const spd_inputs_t& in, const spd_outputs_t& out,
                                               const SurfaceIn& s, const ColScalars& o,
                                               uint32_t neg, int c, int C) {
  const Consts& K = CD.K;
  const bool verify = (K.flags & SPD_FUSE_VERIFY) != 0;
  float* dtp = sm + (size_t)A_DT * KX * kNT + threadIdx.x;
  float* dqp = sm + (size_t)A_DQ * KX * kNT + threadIdx.x;
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
  const bool low = (K.flags & SPD_LOW_LEVEL_WINDS) != 0;
#pragma unroll 4
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    if (!low) {
      __stcs(out.u_wind + i, k == KX - 1 ? o.du_low : 0.0f);
      __stcs(out.v_wind + i, k == KX - 1 ? o.dv_low : 0.0f);
    }
    __stcs(out.temperature + i, dtp[k * kNT]);
    const float dq = dqp[k * kNT];
    __stcs(out.specific_humidity + i, qs != 1.0f ? dq * qs : dq);
  }
  if (low) {  // the lowest level only: single planes
    __stcs(out.u_wind + c, o.du_low);
    __stcs(out.v_wind + c, o.dv_low);
  }
  // diagnostics: stored, or added to the caller's sums under SPD_ACCUMULATE_DIAGNOSTICS
  const bool acc = (K.flags & SPD_ACCUMULATE_DIAGNOSTICS) != 0;
  auto put = [&](float* f, float x) {
    if (f) f[c] = acc ? f[c] + x : x;
  };
  if (acc) {
    out.precnv[c] = out.precnv[c] + o.precnv;
    out.precls[c] = out.precls[c] + o.precls;
  } else {
    __stcs(out.precnv + c, o.precnv);
    __stcs(out.precls + c, o.precls);
  }
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

// The solar row of a column at latitude (sia, coa), finished from the launch's date-only parts
// (Derived): get_zonal_average_fields (shortwave_radiation.py:220-296) with solar (:406-452).
__device__ __forceinline__ ZonalRow zonal_row_of(const Derived& D, float sia, float coa) {
  // clip bounds -1+1e-9 and 1-1e-9 round to -1 and 1 in float32
  const float ch0 = fminf(fmaxf(-D.sol_tdecl * sia / coa, (float)(-1.0 + 1e-9)),
                          (float)(1.0 - 1e-9));
  const float h0 = acosf(ch0);
  const float sh0 = sinf(h0);
  const float fsol = D.sol_scale * (h0 * sia * D.sol_sdecl + sh0 * coa * D.sol_cdecl);
  const float flat2 = 1.5f * (sia * sia) - 0.5f;
  const float ozone = (float)(0.4 * 0.02) * (1.0f + D.coz1 * sia + 1.8f * flat2);
  const float base = 1.0f - (coa * D.cos_rzen + sia * D.sin_rzen);
  const float zenit = 1.0f + base * base;
  ZonalRow r;
  r.fsol = fsol;
  r.ozupp = fsol * 0.01f * zenit;
  r.ozone = fsol * ozone * zenit;
  r.zenit = zenit;
  r.stratz = fmaxf(6.0f - fsol, 0.0f);
  r.sqrt_coa = sqrtf(coa);
  r.pad0 = r.pad1 = 0.0f;
  return r;
}

// The whole column c in one pass: the first half (humidity through clouds) with its level
// arrays in registers, its results and the state moved into the block's shared-memory arena,
// then the second half (radiation, surface fluxes, vertical diffusion) and the outputs.  The
// shortwave uses the level set *S (the instance's, or its prediction); S is read only after the
// first half, behind griddepcontrol.wait (when this launch overlaps the tail of a launch it
// depends on, it waits there for that launch's completion; otherwise it returns at once).
// Returns the column's own cloud-top level bit, 1 << clip(icltop, 0, kx-1).
// The column's inputs are read with the streaming hint (ld.global.cs, evict first), as its
// outputs are written (st.global.cs): each is touched once per call, and a call's hundreds of
// megabytes would otherwise push the kernel's code, its constants and the per-latitude tables
// out of L2 before the next call, whose first wave then fetched them from DRAM (measured with
// per-block start and end times at T425: the first wave's blocks took 31.7 us against 23.6 us in
// steady state, 25.2 us with the hint; the ensemble step went from 0.164 to 0.152 ms and the
// T425 launch from 0.286 to 0.279 ms, results bitwise the same).
// The level-set launch keeps the plain read-only path: the fused launch reads those rows again.
template <int KX>
__device__ __forceinline__ uint32_t fused_process(const ConstsD& CD, float* sm,
                                                  const spd_inputs_t& in,
                                                  const spd_outputs_t& out, const uint32_t* S,
                                                  int c, int C, int il) {
  const Consts& K = CD.K;
  const bool verify = (K.flags & SPD_FUSE_VERIFY) != 0;
  const bool low = (K.flags & SPD_LOW_LEVEL_WINDS) != 0;
  float t[KX], q[KX], phi[KX];
  uint32_t neg = 0;
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    const size_t i = (size_t)k * C + c;
    t[k] = __ldcs(in.temperature + i);
    const float qk = __ldcs(in.specific_humidity + i);
    if (verify && qk < 0.0f) neg |= 1u << k;
    q[k] = (verify && qk < 0.0f) ? 0.0f : qk;
    phi[k] = __ldcs(in.geopotential + i);
  }
  SurfaceIn s;
  s.psa = __ldcs(in.normalized_surface_pressure + c);
  s.fmask = __ldcs(in.fmask + c);
  ColScalars o;
  {
    float qs[KX], dt[KX], dq[KX];
    column_first<KX>(CD, t, q, phi, s, qs, dt, dq, o);
    float* tp = sm + (size_t)A_T * KX * kNT + threadIdx.x;
    float* qp = sm + (size_t)A_Q * KX * kNT + threadIdx.x;
    float* pp = sm + (size_t)A_PHI * KX * kNT + threadIdx.x;
    float* qsp = sm + (size_t)A_QSAT * KX * kNT + threadIdx.x;
    float* dtp = sm + (size_t)A_DT * KX * kNT + threadIdx.x;
    float* dqp = sm + (size_t)A_DQ * KX * kNT + threadIdx.x;
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      tp[k * kNT] = t[k];
      qp[k * kNT] = q[k];
      pp[k * kNT] = phi[k];
      qsp[k * kNT] = qs[k];
      dtp[k * kNT] = dt[k];
      dqp[k * kNT] = dq[k];
    }
  }
  const size_t lw = low ? 0 : (size_t)(KX - 1) * C;
  s.u_low = __ldcs(in.u_wind + lw + c);
  s.v_low = __ldcs(in.v_wind + lw + c);
  s.sst = __ldcs(in.sea_surface_temperature + c);
  s.stl = __ldcs(in.stl_am + c);
  s.soilw = __ldcs(in.soilw_am + c);
  s.snowc = __ldcs(in.snowc_am + c);
  s.sice = __ldcs(in.sice_am + c);
  s.alb0 = __ldcs(in.alb0 + c);
  s.orog = __ldcs(in.orog + c);
  s.phis0 = __ldcs(in.phis0 + c);
  const int j = c % il;
  const ZonalRow z = zonal_row_of(CD.D, __ldg(in.sia + j), __ldg(in.coa + j));
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t Sw = *reinterpret_cast<const volatile uint32_t*>(S);
  column_second<KX>(CD, sm, s, z, Sw, o);
  column_outputs<KX>(CD, sm, in, out, s, o, neg, c, C);
  return 1u << min(max(o.icltop, 0), KX - 1);
}

}  // namespace spd
