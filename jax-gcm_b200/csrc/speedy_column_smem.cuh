// speedy_column_smem.cuh -- the full SPEEDY column, one thread per column, with the per-level
// arrays of each thread in shared memory ([array][level][thread], stride = block size, so a
// warp touching one level of one array hits 32 consecutive banks) and the second half's level
// loops unrolled by 4.  Compared with a fully unrolled register version this keeps the code
// small enough for the instruction cache and the register count low; unrolling by 4 turns the
// shared-memory indices into constant offsets and drops the loop overhead (measured, ragged
// ensemble step 0.199 -> 0.187 ms, T425 call 0.371 -> 0.339 ms; by 2: 0.194 / 0.356 ms;
// 124-126 registers, no spills).  Launch-uniform factors come from Derived (host-evaluated).
//
// Shared memory per thread is the occupancy limit, so only seven level arrays are kept (T, q,
// phi, qsat, the two tendency accumulators and one work array, 56 KB per 128-column block at
// 16 levels -> four blocks per SM): relative humidity is recomputed as q/qsat where used, the
// longwave transmissivities are recomputed in the upward pass, the shortwave and longwave
// absorbed fluxes are added to the temperature accumulator as each piece completes, and the
// vertical-diffusion terms are formed level by level in one ascending pass.
//
// The column is written in two halves: column_first (humidity through clouds) ends at the
// cloud-top level, the one cross-column dependency; column_second (radiation, surface fluxes,
// vertical diffusion) needs the instance's level set of cloud tops and resumes from what the
// first half left (qsat, the tendency accumulators, a few scalars).  The forward runs both in
// one launch (speedy_kernels.cuh, fused_process), with the level set predicted from the
// previous call and checked by the launch's last block (a fixup launch redoes a missed
// instance), or, under SPD_NO_SPECULATION, after a light launch that forms the level set from
// column_first<KX, true>.
//
// Expression order follows the reference term by term (file:line relative to the JAX-GCM
// root).  Deviations, all at the rounding level and never inside a cancelling difference:
// final scalings by 1/psa use one reciprocal, the radiative absorbed-flux pieces of a level are
// scaled and added one at a time instead of summed first, and the second half's exponentials
// (shortwave and longwave transmissivities, the orographic drag factor) use the hardware
// exponential __expf, whose error grows with the argument's magnitude (a few ulp for these
// arguments, which stay within a few units) and leaves the tendencies' distance to the float64
// oracle unchanged at the measured digits.  The saturation humidity keeps expf: it decides
// convection and condensation thresholds.  The forward kernels are compiled with approximate
// division and subnormal flush (jax-gcm_b200/build.py, SOURCE_FLAGS), again with no change in
// the measured distance to the oracles.
#pragma once

#include "speedy_column.cuh"
#include "speedy_derived.h"
#include "speedy_pk.cuh"

namespace spd {

constexpr int kNT = 128;  // threads per block = columns per block

// Exponential of the second half's transmissivities and drag factor: the hardware exponential
// __expf; a build with SPD_IEEE_EXP defined uses expf instead (to measure what the hardware
// exponential changes in the results).
__device__ __forceinline__ float texp(float x) {
#ifdef SPD_IEEE_EXP
  return expf(x);
#else
  return __expf(x);
#endif
}

// Per-thread level array: element k of this thread lives at p[k * kNT].
struct Lv {
  float* p;
  __device__ __forceinline__ float& operator[](int k) const { return p[k * kNT]; }
};

enum { A_T, A_Q, A_PHI, A_QSAT, A_DT, A_DQ, A_W, kNumArrays };

template <int KX>
constexpr size_t smem_bytes() {
  return (size_t)kNumArrays * KX * kNT * sizeof(float);
}


struct ConstsD {
  Consts K;
  Derived D;
};

struct ColScalars {
  float du_low, dv_low, precnv, precls, cbmf, cloudc, clstr, rsds, rsns, ftop_sw, rlds, rlns,
      ftop_lw, tsfc, tskin, shf, evap;
  int iptop, icltop;
};

__device__ __forceinline__ float se_at(const Lv& T, const Lv& PHI, int k) {
  return kCp * T[k] + PHI[k];
}

// Packed pieces of the second half, each a pair of the scalar expressions named beside it (the
// same operations in the same order, so the same bits; checked against those expressions by
// spd_selftest_packed).

// (th(k), th(k - 1)), th(j) = T[j] + wvi[j][1] (T[j + 1] - T[j]) (longwave_radiation.py:49).
__device__ __forceinline__ float2 th_pair(float tkm1, float tk, float tkp1, float wk, float wkm1) {
  const float2 tl = pk(tk, tkm1);
  return pk_add_sep(tl, pk_mul(pk(wk, wkm1), pk_sub(pk(tkp1, tk), tl)));
}

// (st3 t, 4 st3) with st3 = sbc t^3: the blackbody term s0 and the factor of s1
// (longwave_radiation.py:66-68).
__device__ __forceinline__ float2 bb_pair(float t) {
  const float st3 = kSbc * (t * t * t);
  return pk_mul(bc(st3), pk(t, 4.0f));
}

// Shortwave band 1 through a level: (f1, d) = (prev t0 (1 - r), prev (1 - r) (1 - t0))
// (shortwave_radiation.py:124, 137).
__device__ __forceinline__ float2 sw_band1(float prev, float r, float t0) {
  const float2 om = pk_sub(bc(1.0f), pk(r, t0));
  return pk_mul(pk_mul(bc(prev), pk(t0, om.x)), om);
}

// Shortwave band 2 through a level: (prev2 tau1, prev2 (1 - tau1)) (shortwave_radiation.py:141-147).
__device__ __forceinline__ float2 sw_band2(float prev2, float tau1) {
  return pk_mul(bc(prev2), pk(tau1, 1.0f - tau1));
}

// Two absorbed pieces scaled to heating rates: (a g rps, b g rps).
__device__ __forceinline__ float2 sw_scale(float a, float b, float g, float rps) {
  return pk_mul(pk_mul(pk(a, b), bc(g)), bc(rps));
}

// Blackbody emission st4a[k][0..1] (longwave_radiation.py:42-68), from the level temperatures.
template <int KX>
__device__ __forceinline__ void st4a_at(const Consts& K, const Lv& T, int k, float& s0,
                                        float& s1) {
  const spd_vgrid_t& vg = K.vg;
  auto th = [&](int j) { return T[j] + vg.wvi[j][1] * (T[j + 1] - T[j]); };
  if (k == 0) {
    const float x = 0.75f * T[0] + 0.25f * th(0);
    s0 = kSbc * (sq(x) * sq(x));
    s1 = 0.0f;
  } else if (k == 1) {
    const float x = 0.50f * T[1] + 0.25f * (th(0) + th(1));
    s0 = kSbc * (sq(x) * sq(x));
    s1 = 0.0f;
  } else {
    const float t = T[k];
    float grad;
    if (k < KX - 1) {  // th(k) and th(k - 1) as one pair
      const float2 th2 = th_pair(T[k - 1], T[k], T[k + 1], vg.wvi[k][1], vg.wvi[k - 1][1]);
      grad = 0.5f * fmaxf(th2.x - th2.y, 0.0f);
    } else {
      grad = fmaxf(t - th(KX - 2), 0.0f);
    }
    const float2 s04 = bb_pair(t);  // (st3 t, 4 st3)
    s0 = s04.x;
    s1 = s04.y * grad;
  }
}

// s0 of st4a_at alone (the same expressions), for the upward pass, which takes s1 from the
// downward pass.
template <int KX>
__device__ __forceinline__ float st4a_s0(const Consts& K, const Lv& T, int k) {
  if (k <= 1) {
    float s0, s1;
    st4a_at<KX>(K, T, k, s0, s1);
    return s0;
  }
  const float t = T[k];
  const float st3 = kSbc * (t * t * t);
  return st3 * t;
}

// Longwave band energy fractions (radset, longwave_radiation.py:204-226) times (1 - epslw), as
// the band pairs (0, 1) and (2, 3); bands 1 and 2 share their packed quadratic.
__device__ __forceinline__ void radset_w(float temp, float w, float2& fb01, float2& fb23) {
  const float j = fminf(fmaxf(temp, 200.0f), 320.0f);
  const float2 d = pk_sub(bc(j), pk(247.0f, 282.0f));
  const float2 f12 = pk_sub_sep(pk(0.148f, 0.356f), pk_mul(pk(3.0e-6f, 5.2e-6f), pk_mul(d, d)));
  const float f3 = 0.314f + 1.0e-5f * sq(j - 315.0f);
  const float f0 = 1.0f - (((0.0f + f12.x) + f12.y) + f3);
  fb01 = pk_mul(bc(w), pk(f0, f12.x));
  fb23 = pk_mul(bc(w), pk(f12.y, f3));
}

// One band pair's flux recurrence (longwave_radiation.py:99-104 downward, 160-166 upward, the
// sign sg of the gradient term): tau * fl + emis * (fb * (s0 +/- emis * s1)), emis = 1 - tau.
template <bool kDown>
__device__ __forceinline__ float2 lw_step(float2 tau, float2 fl, float2 fb, float s0, float s1) {
  const float2 emis = pk_sub(bc(1.0f), tau);
  const float2 es1 = pk_mul(emis, bc(s1));
  const float2 src = kDown ? pk_add_sep(bc(s0), es1) : pk_sub_sep(bc(s0), es1);
  return pk_add_sep(pk_mul(tau, fl), pk_mul(emis, pk_mul(fb, src)));
}

__device__ __forceinline__ float sum4(float2 a, float2 b) { return ((a.x + a.y) + b.x) + b.y; }

// First half of the column: humidity, convection, large-scale condensation and clouds, with
// every level loop fully unrolled so that the level arrays live in registers.  In: the state T,
// Q (clamped by the caller where verify applies), PHI, and s.psa, s.fmask.  Out: qsat QS, the
// convective + condensation tendency accumulators DT and DQ, and in o the convective and
// cloud results (iptop, icltop, cbmf, precnv, precls, cloudc, clstr).
// kTopOnly: only o.icltop (and o.iptop), from the same expressions, skipping the tendencies,
// precipitation and cloud cover -- the level-set launch, whose S must agree bit for bit with the
// cloud tops the full first half finds.
template <int KX, bool kTopOnly = false>
__device__ __forceinline__ void column_first(const ConstsD& C, const float (&T)[KX],
                                             const float (&Q)[KX], const float (&PHI)[KX],
                                             const SurfaceIn& s, float (&QS)[KX],
                                             float (&DT)[KX], float (&DQ)[KX], ColScalars& o) {
  const Consts& K = C.K;
  const Derived& D = C.D;
  const spd_params_t& p = K.p;
  const spd_vgrid_t& vg = K.vg;
  auto rh_at = [&](int k) { return Q[k] / QS[k]; };  // spec_hum_to_rel_hum (humidity.py:45)
  const float psa = s.psa;
  const float rps = 1.0f / psa;
  float SE[KX];  // dry static energy cp T + phi

  // ---- spec_hum_to_rel_hum (humidity.py:16-51) --------------------------------------------
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    QS[k] = qsat_of(T[k], psa, vg.fsg[k]);
    SE[k] = kCp * T[k] + PHI[k];
  }

  // ---- diagnose_convection (convection.py:15-97) -------------------------------------------
  const float q_b = Q[KX - 1], q_b1 = Q[KX - 2];
  const float se_b = SE[KX - 1], se_b1 = SE[KX - 2];
  int iptop;
  float qdif = 0.0f;
  {
    const float rlhc = (float)(1.0 / 2501.0);
    const float mse0 = se_b + kAlhc * q_b;
    const float mse1 = fminf(mse0, se_b1 + kAlhc * q_b1);
    const float mss0 = fmaxf(mse0, se_b + kAlhc * QS[KX - 1]);
    int ktop1 = KX, ktop2 = KX;
    float msthr = 0.0f;
    float mk1 = SE[KX - 3] + kAlhc * QS[KX - 3];
#pragma unroll
    for (int k = KX - 4; k >= 2; --k) {
      const float mk = SE[k] + kAlhc * QS[k];
      const float mss2 = mk + vg.wvi[k][1] * (mk1 - mk);
      if (mss0 > mss2) ktop1 = k + 1;
      if (mse1 > mss2) {
        ktop2 = k + 1;
        msthr = mss2;
      }
      mk1 = mk;
    }
    const float qthr0 = p.rhbl * QS[KX - 1];
    const float qthr1 = p.rhbl * QS[KX - 2];
    const bool lqthr = (q_b > qthr0) && (q_b1 > qthr1);
    const bool mask_psa = psa > p.psmin;
    const bool case1 = mask_psa && (ktop1 < KX) && (ktop2 < KX);
    const bool case2 = mask_psa && (ktop1 < KX) && !(ktop2 < KX) && lqthr;
    if (case1) qdif = fmaxf(q_b - qthr0, (mse0 - msthr) * rlhc);
    if (case2) qdif = q_b - qthr0;
    iptop = (case1 || case2) ? ktop1 : KX + 1;
  }

  // ---- get_convection_tendencies (convection.py:99-237) -----------------------------------
  if constexpr (!kTopOnly) {
    const bool mask = iptop < KX;
    const float qmax = fmaxf(1.01f * q_b, QS[KX - 1]);
    const float w_last = vg.wvi[KX - 2][1];
    const float sb = se_b1 + w_last * (se_b - se_b1);
    const float qb = fminf(q_b1 + w_last * (q_b - q_b1), q_b);
    const float fpsa = psa * fminf(1.0f, (psa - p.psmin) * D.rdps);
    const float fmass = D.fm0 * fpsa * fminf(5.0f, qdif / (qmax - qb));
    const float cbmf = mask ? fmass : 0.0f * fmass;
    const float fus = fmass * se_b, fuq = fmass * qmax;
    const float fds = fmass * sb, fdq = fmass * qb;
    float cm = 0.0f, cs = 0.0f, cq = 0.0f, fsq_sum = 0.0f;
    float fm_n = 0.f, fus_n = 0.f, fuq_n = 0.f, fds_n = 0.f, fdq_n = 0.f;
    float dfqa_last = 0.0f, precnv = 0.0f;
    float se_k = se_b, q_k = q_b;
#pragma unroll
    for (int k = KX - 1; k >= 0; --k) {
      const bool lm = (k <= KX - 2) && (k >= iptop);
      float en = (k >= 1 && k <= KX - 2) ? D.entr[k] * psa * cbmf : 0.0f;
      en = lm ? en : 0.0f * en;
      cm = cm + en * 1.0f;
      cs = cs + en * se_k;
      cq = cq + en * q_k;
      const float fm_k = fmass + cm, fus_k = fus + cs, fuq_k = fuq + cq;
      float se_m = 0.0f, q_m = 0.0f, fds_k, fdq_k;
      if (k >= 1) {
        se_m = SE[k - 1];
        q_m = Q[k - 1];
      }
      if (k == KX - 1) {
        fds_k = fds;
        fdq_k = fdq;
      } else {
        const float w = (k >= 1) ? vg.wvi[k - 1][1] : 0.0f;
        const float sb3 = (k >= 1) ? se_m + w * (se_k - se_m) : 0.0f;
        const float qb3 = (k >= 1) ? q_m + w * (q_k - q_m) : 0.0f;
        fds_k = fm_k * sb3;
        fdq_k = fm_k * qb3;
      }
      float dfse, dfqa;
      if (k == KX - 1) {
        dfse = fds - fus;
        dfqa = fdq - fuq;
      } else {
        const float a = (fus_n - fds_n) - (fus_k - fds_k);
        const float b = (fuq_n - fdq_n) - (fuq_k - fdq_k);
        dfse = lm ? a : 0.0f * a;
        dfqa = lm ? b : 0.0f * b;
      }
      const float dq0 = p.rhil * QS[k] - q_k;
      const float delq = lm ? dq0 : 0.0f * dq0;
      const float fsq = (delq > 0.0f ? p.smf : 0.0f * p.smf) * cbmf * delq;
      dfqa = dfqa + fsq;
      fsq_sum = fsq_sum + fsq;
      if (k == iptop - 1) {
        // top layer (detrainment, precipitation), fluxes taken at level iptop = k + 1
        const float qsatb = QS[k] + vg.wvi[k][1] * (QS[k + 1] - QS[k]);
        precnv = fmaxf(fuq_n - fm_n * qsatb, 0.0f);
        dfse = fus_n - fds_n + kAlhc * precnv;
        dfqa = fuq_n - fdq_n - precnv;
      }
      if (k == KX - 1) {
        dfqa_last = dfqa;
        DT[k] = dfse * rps * vg.grdscp[k];
      } else if (k == 0) {
        DT[0] = dfse;
        DQ[0] = dfqa;
      } else {
        DT[k] = dfse * rps * vg.grdscp[k];
        DQ[k] = dfqa * rps * vg.grdsig[k];
      }
      fm_n = fm_k;
      fus_n = fus_k;
      fuq_n = fuq_k;
      fds_n = fds_k;
      fdq_n = fdq_k;
      se_k = se_m;
      q_k = q_m;
    }
    DQ[KX - 1] = (dfqa_last + (-fsq_sum)) * rps * vg.grdsig[KX - 1];
    o.cbmf = cbmf;
    o.precnv = precnv;
  }

  // ---- get_large_scale_condensation_tendencies (large_scale_condensation.py:14-86) --------
  {
    const float tfact = (float)(2501.0 / 1004.0);
    const float psa2 = psa * psa;
    float psum = 0.0f;
    int first = 0;
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      const float dqa = D.rhref[k] * QS[k] - Q[k];
      float dql = 0.0f, dtl = 0.0f;
      if (dqa < 0.0f) {
        dql = dqa * D.rtlsc;
        dtl = tfact * fminf(-dql, D.dqmax[k] * psa2);
        if (first == 0) first = k;
      }
      if constexpr (!kTopOnly) {
        DT[k] = DT[k] + dtl;
        DQ[k] = DQ[k] + dql;
        psum = psum + D.pfact[k] * dql;
      }
    }
    if constexpr (!kTopOnly) o.precls = (0.0f - psum) * psa;
    iptop = min(first == 0 ? 1 : first, iptop);
  }
  o.iptop = iptop;

  // ---- clouds (shortwave_radiation.py:313-404) ---------------------------------------------
  float cloudc, clstr, qcloud;
  int icltop;
  {
    const int nl1 = KX - 2;
    const float rh_nl1 = rh_at(nl1);
    const bool m0 = rh_nl1 > p.rhcl1;
    const float cloudc0 = m0 ? rh_nl1 - p.rhcl1 : 0.0f;
    const int icl0 = m0 ? nl1 : KX;
    // Lines 365-373 take, over k = 2..kx-3, the max of (cmax == upd_k ? (m_k ? k : icl0) : icl0)
    // with icl0 >= kx-2 > k.  That max is kx-3 exactly when every level has m_k and
    // upd_k == cmax (i.e. all m_k and min upd == max upd), and icl0 otherwise: one pass.
    float cmax = -INFINITY, cmin = INFINITY;
    bool allm = true;
#pragma unroll
    for (int k = 2; k < KX - 2; ++k) {
      const float drh = rh_at(k) - p.rhcl1;
      const bool m = (drh > cloudc0) && (Q[k] > p.qacl);
      const float upd = m ? drh : cloudc0;
      cmax = fmaxf(cmax, upd);
      cmin = fminf(cmin, upd);
      allm = allm && m;
    }
    const int icl = (allm && cmin == cmax) ? KX - 3 : icl0;
    if constexpr (kTopOnly) {
      o.icltop = min(iptop, icl);
      return;
    }
    const float gse = (se_b1 - se_b) / (PHI[KX - 2] - PHI[KX - 1]);
    const float pr1 = fminf(p.pmaxcl, 86.4f * (o.precnv + o.precls));
    cloudc = fminf(1.0f, p.wpcl * sqrtf(fmaxf(kEpsilon, pr1)) + sq(fminf(1.0f, cmax * D.rrcl)));
    if (isnan(cloudc)) cloudc = 1.0f;
    icltop = min(iptop, icl);
    qcloud = Q[nl1];
    const float fstab = fminf(fmaxf(D.rgse * (gse - p.gse_s0), 0.0f), 1.0f);
    clstr = fstab * fmaxf(p.clsmax - 1.2f * cloudc, 0.0f);
    const float clstrl = fmaxf(clstr, p.clsminl) * rh_at(KX - 1);
    clstr = clstr + s.fmask * (clstrl - clstr);
  }
  o.cloudc = cloudc;
  o.clstr = clstr;
  o.icltop = icltop;
}

// Second half: shortwave, longwave, surface fluxes and vertical diffusion, from the state, qsat
// and tendency accumulators in shared memory and the first half's results in o.
template <int KX>
__device__ void column_second(const ConstsD& C, float* sm, const SurfaceIn& s, const ZonalRow& z,
                              uint32_t S, ColScalars& o) {
  const Consts& K = C.K;
  const Derived& D = C.D;
  const spd_params_t& p = K.p;
  const spd_vgrid_t& vg = K.vg;
  const int tid = threadIdx.x;
  auto arr = [&](int a) { return Lv{sm + (size_t)a * KX * kNT + tid}; };
  const Lv T = arr(A_T), Q = arr(A_Q), PHI = arr(A_PHI), QS = arr(A_QSAT), DT = arr(A_DT),
           DQ = arr(A_DQ), W = arr(A_W);
  auto rh_at = [&](int k) { return Q[k] / QS[k]; };  // spec_hum_to_rel_hum (humidity.py:45)
  const float psa = s.psa;
  const float rps = 1.0f / psa;
  const float snowc = fminf(1.0f, s.snowc);
  const float alb_l = s.alb0 + snowc * (p.albsn - s.alb0);
  const float alb_s = p.albsea + s.sice * (p.albice - p.albsea);
  const float albsfc = alb_s + s.fmask * (alb_l - alb_s);
  const float q_b = Q[KX - 1];
  const float se_b = se_at(T, PHI, KX - 1), se_b1 = se_at(T, PHI, KX - 2);
  const int iptop = o.iptop;
  const float cloudc = o.cloudc, clstr = o.clstr, qcloud = Q[KX - 2];
  const int icltop = o.icltop;

  // ---- shortwave_rad_fluxes (shortwave_radiation.py:27-217); W = reflection tau2[:,2] -------
  float flux_sw0, flux_sw1, rsds;
  {
    const bool cmask = icltop < KX;
    const float refl = cmask ? p.albcl * cloudc : 0.0f;
    const float psaz = psa * z.zenit;
    const float acloud = cloudc * fminf(p.abscl1 * qcloud, p.abscl2);
    const bool gate = (K.model_step % 3) == 0;
    // band-1 transmissivity of level k (lines 80-94)
    auto tau0_at = [&](int k) {
      if (k == 0) return texp(-psaz * vg.dhs[0] * p.absdry);
      const float cl = (k >= icltop && k < KX - 1) ? acloud : 0.0f;
      return texp(-psaz * vg.dhs[k] * (D.abs1[k] + p.abswv1 * Q[k] + cl));
    };
    auto add_sw = [&](int k, float d) { DT[k] = DT[k] + (gate ? d * vg.grdscp[k] * rps : 0.0f); };
#pragma unroll 4
    for (int k = 0; k < KX - 1; ++k) W[k] = ((S >> k) & 1u) ? refl : 0.0f;
    W[KX - 1] = p.albcls * clstr;
    const float fband2 = 0.05f, fband1 = 0.95f;
    float f1 = z.fsol * fband1;
    float d0 = f1;
    f1 = tau0_at(0) * (f1 - z.ozupp * psa);
    add_sw(0, d0 + (-f1));
    d0 = f1;
    f1 = tau0_at(1) * (f1 - z.ozone * psa);
    const float d1_band1 = d0 + (-f1);
    float f2 = z.fsol * fband2;
    {  // band 2 at level 1 completes level 1's downward absorption
      const float tau1 = texp(-psaz * vg.dhs[1] * p.abswv2 * Q[1]);
      const float prev = f2;
      f2 = prev * tau1;
      add_sw(1, d1_band1);
      add_sw(1, prev * (1.0f - tau1));
    }
    // Levels 2..kx-1, two bands and two absorbed pieces in packed pairs: the exponents
    // (m x_k, m abswv2) with m = -psaz dhs_k, then (prev t0, prev (1 - r)) x ((1 - r), (1 - t0))
    // = (f1, d), (prev2 tau1, prev2 (1 - tau1)), and both pieces' scalings.
#pragma unroll 4
    for (int k = 2; k < KX; ++k) {
      const float prev = f1, r = W[k];
      const float cl = (k < KX - 1 && k >= icltop) ? acloud : 0.0f;
      const float m = -psaz * vg.dhs[k];
      const float2 ex = pk_mul(bc(m), pk(D.abs1[k] + p.abswv1 * Q[k] + cl, p.abswv2));
      const float t0 = texp(ex.x), tau1 = texp(ex.y * Q[k]);
      const float2 fd = sw_band1(prev, r, t0);
      f1 = fd.x;
      W[k] = r * prev;
      const float prev2 = f2;
      const float2 f2e = sw_band2(prev2, tau1);
      f2 = f2e.x;
      const float2 g = sw_scale(fd.y, f2e.y, vg.grdscp[k], rps);
      DT[k] = (DT[k] + (gate ? g.x : 0.0f)) + (gate ? g.y : 0.0f);
    }
    rsds = f1 + f2;
    float up = f1 * albsfc;
    o.rsns = rsds - up;
    float t_k = tau0_at(KX - 1);
    add_sw(KX - 1, up * (1.0f - t_k));
#pragma unroll 4
    for (int k = KX - 1; k >= 1; --k) {
      up = up * t_k + W[k];
      t_k = tau0_at(k - 1);
      add_sw(k - 1, up * (1.0f - t_k));
    }
    const float ftop_up = t_k * up + W[0];
    o.ftop_sw = z.fsol - ftop_up;
    flux_sw0 = ftop_up;
    flux_sw1 = f2;
  }
  o.rsds = rsds;

  // ---- longwave transmissivities of level k (shortwave_radiation.py:174-206) ---------------
  const float acl1 = cloudc * p.ablcl1, acl2 = cloudc * p.ablcl2;
  // (-a * psa) * dhs, formed as -((a * psa) * dhs): the same bits (round-to-nearest is
  // symmetric in sign)
  auto lw_tau = [&](int k, float2& t01, float2& t23) {
    float2 a23 = pk_mul(pk(p.ablwv1, p.ablwv2), bc(Q[k]));
    float a0 = p.ablwin;
    if (k == 0) a23 = bc(0.0f);
    if (k >= 2 && k <= KX - 2) {
      a0 = a0 + ((k > icltop) ? acl1 : acl2);
      a23 = pk(fmaxf(a23.x, acl2), fmaxf(a23.y, acl2));
    }
    const float2 pd = bc(vg.dhs[k]);
    const float2 x01 = pk_mul(pk_mul(pk(a0, D.ablco2), bc(psa)), pd);
    const float2 x23 = pk_mul(pk_mul(a23, bc(psa)), pd);
    t01 = pk(texp(-x01.x), texp(-x01.y));
    t23 = pk(texp(-x23.x), texp(-x23.y));
  };
  auto add_lw = [&](int k, float d) { DT[k] = DT[k] + d * vg.grdscp[k] * rps; };

  // ---- get_downward_longwave_rad_fluxes (longwave_radiation.py:13-117) ---------------------
  float rlds;
  {
    // W keeps each level's blackbody gradient term s1 for the upward pass (W is free once the
    // shortwave is done)
    float2 fl01, fl23, fb01, fb23, t01, t23;
    float s0, s1;
    st4a_at<KX>(K, T, 0, s0, s1);
    radset_w(T[0], D.w_lw, fb01, fb23);
    lw_tau(0, t01, t23);
    {  // the top level: no flux from above; bands 2 and 3 start at zero
      const float2 emis = pk_sub(bc(1.0f), t01);
      fl01 = pk_mul(emis, pk_mul(fb01, pk_add_sep(bc(s0), pk_mul(emis, bc(s1)))));
      fl23 = bc(0.0f);
    }
    float sprev = sum4(fl01, fl23);
    add_lw(0, 0.0f + (-sprev));
#pragma unroll 4
    for (int k = 1; k < KX; ++k) {
      st4a_at<KX>(K, T, k, s0, s1);
      W[k] = s1;
      radset_w(T[k], D.w_lw, fb01, fb23);
      lw_tau(k, t01, t23);
      fl01 = lw_step<true>(t01, fl01, fb01, s0, s1);
      fl23 = lw_step<true>(t23, fl23, fb23, s0, s1);
      const float sk = sum4(fl01, fl23);
      float d = 0.0f + (-(sk - sprev));
      if (k == KX - 1) d = d + (-(D.corlw_f * s0));
      add_lw(k, d);
      sprev = sk;
    }
    rlds = sum4(pk_mul(bc(p.emisfc), fl01), pk_mul(bc(p.emisfc), fl23));
    rlds = rlds + D.corlw_f * s0;
  }
  o.rlds = rlds;

  // ---- get_surface_fluxes (surface_flux.py:15-300) ----------------------------------------
  float rlus2 = 0.0f, tsfc = 0.0f, tskin_out = 0.0f;
  {
    const float ta1 = T[KX - 1], ta2 = T[KX - 2];
    const float ua = s.u_low, va = s.v_low;
    const float phi0 = s.orog * kGrav;
    const float u0 = p.fwind0 * ua, v0 = p.fwind0 * va;
    float ustr0 = 0.f, ustr1 = 0.f, vstr0 = 0.f, vstr1 = 0.f, shf0 = 0.f;
    float evap0 = 0.f, rlus0 = 0.f;
    float t1_1 = 0.f, q1_1 = 0.f, denv2 = 0.f, tskin = 0.f;
    const bool land = (K.flags & SPD_LFLUXLAND) != 0;
    if (land) {
      const float rcp = (float)(1.0 / 1004.0);
      const float dt1 = vg.wvi[KX - 1][1] * (ta1 - ta2);
      float t1_0 = 0.0f + (ta1 + dt1);
      t1_1 = t1_0 - phi0 * dt1 / D.rgas288_sigl;
      const float t2_1 = ta1 + rcp * PHI[KX - 1];
      const float t2_0 = t2_1 - rcp * phi0;
      if (ta1 > ta2) {
        t1_0 = p.ftemp0 * t1_0 + D.gtemp0 * t2_0;
        t1_1 = p.ftemp0 * t1_1 + D.gtemp0 * t2_1;
      } else {
        t1_0 = ta1;
        t1_1 = ta1;
      }
      const float t0 = t1_1 + s.fmask * (t1_0 - t1_1);
      const float denv0 =
          (kP0 * psa / (kRgas * t0)) * sqrtf(u0 * u0 + v0 * v0 + p.vgust * p.vgust);
      tskin = s.stl + p.ctday * z.sqrt_coa * rsds * (1.0f - alb_l) * psa;
      const float dthl = (tskin > t2_0) ? fminf(p.dtheta, tskin - t2_0)
                                        : fmaxf(-p.dtheta, D.astab * (tskin - t2_0));
      const float denv1 = denv0 * (1.0f + dthl * D.rdth);
      const float forog = 1.0f + D.rhdrag * (1.0f - texp(-fmaxf(s.phis0, 0.0f) * D.rhdrag));
      const float cdldv = p.cdl * denv0 * forog;
      ustr0 = -cdldv * ua;
      vstr0 = -cdldv * va;
      shf0 = D.chlcp * denv1 * (tskin - t1_0);
      const float q1_0 = (p.fhum0 > 0.0f)
                             ? p.fhum0 * (rh_at(KX - 1) * qsat_of(t1_0, psa, 1.0f)) + D.ghum0 * q_b
                             : q_b;
      const float qs00 = qsat_of(tskin, psa, 1.0f);
      evap0 = p.chl * denv1 * fmaxf(0.0f, s.soilw * qs00 - q1_0);
      const float tsk3 = tskin * tskin * tskin;
      const float drls = 4.0f * D.esbc * tsk3;
      rlus0 = D.esbc * tsk3 * tskin;
      float hfl0 = rsds * (1.0f - alb_l) + rlds - (rlus0 + shf0 + (kAlhc * evap0));
      if (K.flags & SPD_LSKINEB) {
        const float clamb = p.clambda + (snowc * (p.clambsn - p.clambda));
        hfl0 = hfl0 - (clamb * (tskin - s.stl));
        float qs01 = qsat_of(tskin + 1.0f, psa, 1.0f);
        qs01 = (evap0 > 0.0f) ? s.soilw * (qs01 - qs00) : 0.0f;
        const float dtskin = hfl0 / (clamb + drls + (p.chl * denv1 * (kCp + (kAlhc * qs01))));
        tskin = tskin + dtskin;
        shf0 = shf0 + D.chlcp * denv1 * dtskin;
        evap0 = evap0 + p.chl * denv1 * qs01 * dtskin;
        rlus0 = rlus0 + drls * dtskin;
      }
      const float sst = s.sst;
      const float dths = (sst > t2_1) ? fminf(p.dtheta, sst - t2_1)
                                      : fmaxf(-p.dtheta, D.astab * (sst - t2_1));
      denv2 = denv0 * (1.0f + dths * D.rdth);
      q1_1 = (p.fhum0 > 0.0f)
                 ? p.fhum0 * (rh_at(KX - 1) * qsat_of(t1_1, psa, 1.0f)) + D.ghum0 * q_b
                 : q_b;
      const float cdsdv = p.cds * denv2;
      ustr1 = -cdsdv * ua;
      vstr1 = -cdsdv * va;
    }
    const float sst = s.sst;
    const float shf1 = p.chs * kCp * denv2 * (sst - t1_1);
    const float evap1 = p.chs * denv2 * (qsat_of(sst, psa, 1.0f) - q1_1);
    const float rlus1 = D.esbc * (sq(sst) * sq(sst));
    float ustr2 = 0.f, vstr2 = 0.f, shf2 = 0.f, evap2 = 0.f;
    if (land) {
      const float fm = s.fmask;
      ustr2 = ustr1 + fm * (ustr0 - ustr1);
      vstr2 = vstr1 + fm * (vstr0 - vstr1);
      shf2 = shf1 + fm * (shf0 - shf1);
      evap2 = evap1 + fm * (evap0 - evap1);
      rlus2 = rlus1 + fm * (rlus0 - rlus1);
      tsfc = sst + fm * (s.stl - sst);
      tskin_out = sst + fm * (tskin - sst);
    }
    o.du_low = 0.0f + ustr2 * rps * vg.grdsig[KX - 1];
    o.dv_low = 0.0f + vstr2 * rps * vg.grdsig[KX - 1];
    DT[KX - 1] = DT[KX - 1] + (0.0f + shf2 * rps * vg.grdscp[KX - 1]);
    DQ[KX - 1] = DQ[KX - 1] + (0.0f + evap2 * rps * vg.grdsig[KX - 1]);
    o.shf = shf2;
    o.evap = evap2;
  }
  o.tsfc = tsfc;
  o.tskin = tskin_out;

  // ---- get_upward_longwave_rad_fluxes (longwave_radiation.py:119-202) ---------------------
  {
    o.rlns = rlus2 - rlds;
    float2 fb01, fb23, fl01, fl23, t01, t23;
    float s0, s1;
    radset_w(tsfc, D.w_lw, fb01, fb23);
    fl01 = pk_add_sep(pk_mul(fb01, bc(rlus2)), pk_mul(bc(D.refsfc), pk(flux_sw0, flux_sw1)));
    fl23 = pk_add_sep(pk_mul(fb23, bc(rlus2)), pk_mul(bc(D.refsfc), bc(0.0f)));
    float sk = sum4(fl01, fl23);
    float d_last = p.epslw * rlus2;  // dfabs[kx-1] += epslw*rlus before the scan
#pragma unroll 4
    for (int k = KX - 1; k >= 1; --k) {
      s0 = st4a_s0<KX>(K, T, k);
      s1 = W[k];
      radset_w(T[k], D.w_lw, fb01, fb23);
      lw_tau(k, t01, t23);
      fl01 = lw_step<false>(t01, fl01, fb01, s0, s1);
      fl23 = lw_step<false>(t23, fl23, fb23, s0, s1);
      const float skm1 = sum4(fl01, fl23);
      float d = (sk - skm1);
      if (k == KX - 1) d = d_last + d;
      if (k >= 2) add_lw(k, d);
      else d_last = d;  // level 1 still gets -corlw2
      sk = skm1;
    }
    st4a_at<KX>(K, T, 0, s0, s1);
    float s0b, s1b;
    st4a_at<KX>(K, T, 1, s0b, s1b);
    radset_w(T[0], D.w_lw, fb01, fb23);
    lw_tau(0, t01, t23);
    const float2 top01 = lw_step<false>(t01, fl01, fb01, s0, s1);  // bands 2, 3 pass level 0
    const float stratc0 = z.stratz * psa, stratc1 = D.eps1 * psa;
    const float corlw1 = vg.dhs[0] * stratc1 * s0 + stratc0;
    const float corlw2 = vg.dhs[1] * stratc1 * s0b;
    const float2 dtop = pk_sub(fl01, top01);
    add_lw(0, (dtop.x + dtop.y) + (-corlw1));
    add_lw(1, d_last + (-corlw2));
    o.ftop_lw = (corlw1 + corlw2) + sum4(top01, fl23);
  }

  // ---- get_vertical_diffusion_tend (vertical_diffusion.py:10-136) -------------------------
  // Each level's ttenvd / qtenvd is formed completely, in the reference's order, and then added
  // to the accumulated tendency (total + ttenvd, speedy_physics.py:125).  The "-" updates of
  // lines 118 and 131 reach level k one step after its "+" update, so one ascending pass
  // carries them in a register.
  {
    const int nl1 = KX - 1;
    const int icnv = KX - iptop - 1;
    const float rh_b = rh_at(KX - 1), rh_b1 = rh_at(nl1 - 1);
    const float dmse = se_b - se_b1 + kAlhc * (q_b - QS[nl1 - 1]);
    const float drh = rh_b - rh_b1;
    const float fcnv = (icnv > 0 && dmse >= 0.0f) ? p.redshc : 1.0f;
    float tt_sh1 = 0.0f, tt_sh0 = 0.0f, qt_sh1 = 0.0f, qt_sh0 = 0.0f;  // levels kx-2, kx-1
    if (dmse >= 0.0f) {
      const float fluxse = fcnv * D.fshcse * dmse;
      tt_sh1 = fluxse * D.rsig[nl1 - 1];
      tt_sh0 = -fluxse * D.rsig[KX - 1];
      if (drh >= 0.0f) {
        const float fq = fcnv * D.fshcq * QS[KX - 1] * drh;
        qt_sh1 = fq * D.rsig[nl1 - 1];
        qt_sh0 = -fq * D.rsig[KX - 1];
      }
    } else if (dmse < 0.0f && drh > D.drh0) {
      const float fq = D.fvdiq2 * QS[nl1 - 1] * drh;
      qt_sh1 = fq * D.rsig[nl1 - 1];
      qt_sh0 = -fq * D.rsig[KX - 1];
    }
    // moisture diffusion above the PBL (lines 99-118), levels 2..kx-3 and the "-" at kx-2
    float pend = 0.0f;
    float rh_k = rh_at(2);
#pragma unroll 4
    for (int k = 2; k < KX - 2; ++k) {
      const float rh_n = rh_at(k + 1);
      const float dr = rh_n - rh_k;
      const bool cond = (D.vdcond >> k) & 1u;
      const float fq = (dr >= D.drh0v[k] && cond) ? D.fvdiq2v[k] * QS[k] * dr : 0.0f;
      const float2 fr = pk_mul(bc(fq), pk(D.rsig[k], D.rsig[k + 1]));
      const float qk = (k == 2) ? (0.0f + fr.x) : (0.0f + fr.x) + pend;
      DQ[k] = DQ[k] + qk;
      pend = -fr.y;
      rh_k = rh_n;
    }
    DQ[KX - 2] = DQ[KX - 2] + (qt_sh1 + pend);
    DQ[KX - 1] = DQ[KX - 1] + qt_sh0;
    // damping of super-adiabatic lapse rate (lines 121-131)
    float cum = 0.0f;
    float se_k = se_at(T, PHI, 0), phi_k = PHI[0];
    float pend_t = 0.0f;
#pragma unroll 4
    for (int k = 0; k < nl1; ++k) {
      const float se_n = se_at(T, PHI, k + 1), phi_n = PHI[k + 1];
      const float se0 = se_n - p.segrad * (phi_n - phi_k);
      const float fse = (se_k < se0) ? D.fvdise * (se0 - se_k) : 0.0f;
      const float base = (k == KX - 2) ? tt_sh1 : 0.0f;
      const float2 fr = pk_mul(bc(fse), pk(D.rsig[k], D.rsig1[k]));
      const float tk = (k == 0) ? (base + fr.x) : (base + fr.x) + pend_t;
      DT[k] = DT[k] + tk;
      cum = cum + fr.y;
      pend_t = -cum;
      se_k = se_n;
      phi_k = phi_n;
    }
    DT[KX - 1] = DT[KX - 1] + (tt_sh0 + pend_t);
  }
}

}  // namespace spd
