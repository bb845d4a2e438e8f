// speedy_column.cuh -- SPEEDY column physics for one grid column, evaluated by one thread.
//
// Each stage restates one reference term (file:line relative to the JAX-GCM root) and keeps
// its float32 expression order, so results agree with the reference's float32 arithmetic to
// rounding.  Level arrays are template-sized (KX = 7, 8 or 16) and fully unrolled so that they
// live in registers.  Python double constants that the reference combines with float32 data
// are rounded to float32 exactly as JAX's weak typing does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "speedy_b200.h"

namespace spd {

// jcm/constants.py:3-5, physics/speedy/physical_constants.py:9-45
constexpr double kRgasD = 2.0 / 7.0 * 1004.0;
constexpr float kP0 = 1e5f;
constexpr float kGrav = 9.81f;
constexpr float kCp = 1004.0f;
constexpr float kRgas = (float)kRgasD;
constexpr float kAlhc = 2501.0f;
constexpr float kSbc = (float)5.67e-8;
constexpr float kEpsilon = (float)1e-9;

// Per-latitude solar table row (get_zonal_average_fields, shortwave_radiation.py:220-296),
// plus sqrt(coa) for the skin temperature (surface_flux.py:132).
struct alignas(32) ZonalRow {
  float fsol, ozupp, ozone, zenit, stratz, sqrt_coa, pad0, pad1;
};

// Launch-invariant inputs passed by value.
struct Consts {
  spd_vgrid_t vg;
  spd_params_t p;
  int C;          // columns = ix * il
  int il;
  uint32_t flags;
  float tyear;
  int model_year, model_step, co2_year_ref;
  float dt_seconds, q_tend_scale;
};

__device__ __forceinline__ float sq(float x) { return x * x; }

// get_qsat (humidity.py:73-104) for sig > 0.
__device__ __forceinline__ float qsat_of(float ta, float ps, float sig) {
  const float e0 = 6.108e-3f, c1 = 17.269f, c2 = 21.875f, t0 = 273.16f, t1 = 35.86f,
              t2 = 7.66f;
  float e = (ta >= t0) ? e0 * expf(c1 * (ta - t0) / (ta - t1))
                       : e0 * expf(c2 * (ta - t0) / (ta - t2));
  return 622.0f * e / (sig * ps - 0.378f * e);
}

// radset (longwave_radiation.py:204-226): band energy fractions times (1 - epslw).
__device__ __forceinline__ void radset(float temp, float epslw, float fb[4]) {
  float j = fminf(fmaxf(temp, 200.0f), 320.0f);
  float f1 = 0.148f - 3.0e-6f * sq(j - 247.0f);
  float f2 = 0.356f - 5.2e-6f * sq(j - 282.0f);
  float f3 = 0.314f + 1.0e-5f * sq(j - 315.0f);
  float f0 = 1.0f - (((0.0f + f1) + f2) + f3);
  float w = 1.0f - epslw;
  fb[0] = w * f0;
  fb[1] = w * f1;
  fb[2] = w * f2;
  fb[3] = w * f3;
}

__device__ __forceinline__ float sum4(const float a[4]) { return ((a[0] + a[1]) + a[2]) + a[3]; }

// solar (shortwave_radiation.py:406-452) for one latitude, csol = 4*solc.
__device__ __forceinline__ float solar_topsr(float tyear, float sia, float coa) {
  const float pigr = 2.0f * asinf(1.0f);
  float alpha = 2.0f * pigr * tyear;
  float ca1 = cosf(alpha), sa1 = sinf(alpha);
  float ca2 = ca1 * ca1 - sa1 * sa1;
  float sa2 = 2.0f * sa1 * ca1;
  float ca3 = ca1 * ca2 - sa1 * sa2;
  float sa3 = sa1 * ca2 + sa2 * ca1;
  float decl = 0.006918f - 0.399912f * ca1 + 0.070257f * sa1 - 0.006758f * ca2 +
               0.000907f * sa2 - 0.002697f * ca3 + 0.001480f * sa3;
  float fdis = 1.000110f + 0.034221f * ca1 + 0.001280f * sa1 + 0.000719f * ca2 + 0.000077f * sa2;
  float cdecl = cosf(decl), sdecl = sinf(decl);
  float tdecl = sdecl / cdecl;
  float csolp = 1368.0f / pigr;
  // clip bounds -1+1e-9 and 1-1e-9 round to -1 and 1 in float32
  float ch0 = fminf(fmaxf(-tdecl * sia / coa, (float)(-1.0 + 1e-9)), (float)(1.0 - 1e-9));
  float h0 = acosf(ch0);
  float sh0 = sinf(h0);
  return csolp * fdis * (h0 * sia * sdecl + sh0 * coa * cdecl);
}

// get_zonal_average_fields (shortwave_radiation.py:220-296) for latitude j.
__device__ __forceinline__ ZonalRow zonal_row(float tyear, float sia, float coa) {
  const float asin1 = asinf(1.0f);
  float alpha = 4.0f * asin1 * (tyear + (float)(10.0 / 365.0));
  float coz1 = fmaxf(0.0f, cosf(alpha - 0.0f));
  float rzen = -cosf(alpha) * 23.45f * asin1 / 90.0f;
  float fsol = solar_topsr(tyear, sia, coa);
  float flat2 = 1.5f * (sia * sia) - 0.5f;
  float ozone = (float)(0.4 * 0.02) * (1.0f + coz1 * sia + 1.8f * flat2);
  float base = 1.0f - (coa * cosf(rzen) + sia * sinf(rzen));
  float zenit = 1.0f + base * base;
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

// ---------------------------------------------------------------------------------------------
// Stages shared by the cloud-top pre-pass and the full column.
// ---------------------------------------------------------------------------------------------

// diagnose_convection (convection.py:15-97).  Returns iptop; qdif through the reference.
template <int KX>
__device__ __forceinline__ int diagnose_convection(const Consts& K, const float se[KX],
                                                   const float q[KX], const float qsat[KX],
                                                   float psa, float& qdif) {
  const spd_params_t& p = K.p;
  const float rlhc = (float)(1.0 / 2501.0);
  float mse0 = se[KX - 1] + kAlhc * q[KX - 1];
  float mse1 = fminf(mse0, se[KX - 2] + kAlhc * q[KX - 2]);
  float mss_last = se[KX - 1] + kAlhc * qsat[KX - 1];
  float mss0 = fmaxf(mse0, mss_last);
  int ktop1 = KX, ktop2 = KX;
  float msthr = 0.0f;  // mss2[kx-1] padding value
  // levels 2 .. kx-4, first unstable from the top
#pragma unroll
  for (int k = KX - 4; k >= 2; --k) {
    float mk = se[k] + kAlhc * qsat[k];
    float mk1 = se[k + 1] + kAlhc * qsat[k + 1];
    float mss2 = mk + K.vg.wvi[k][1] * (mk1 - mk);
    if (mss0 > mss2) ktop1 = k + 1;
    if (mse1 > mss2) {
      ktop2 = k + 1;
      msthr = mss2;
    }
  }
  float qthr0 = p.rhbl * qsat[KX - 1];
  float qthr1 = p.rhbl * qsat[KX - 2];
  bool lqthr = (q[KX - 1] > qthr0) && (q[KX - 2] > qthr1);
  bool mask_psa = psa > p.psmin;
  bool case1 = mask_psa && (ktop1 < KX) && (ktop2 < KX);
  bool case2 = mask_psa && (ktop1 < KX) && !(ktop2 < KX) && lqthr;
  qdif = 0.0f;
  if (case1) qdif = fmaxf(q[KX - 1] - qthr0, (mse0 - msthr) * rlhc);
  if (case2) qdif = q[KX - 1] - qthr0;
  return (case1 || case2) ? ktop1 : KX + 1;
}

// First level k >= 1 with rhref*qsat - q < 0, else 1 (large_scale_condensation.py:74).
template <int KX>
__device__ __forceinline__ int lsc_top(const Consts& K, const float q[KX], const float qsat[KX]) {
  int first = 1;
  bool found = false;
#pragma unroll
  for (int k = 1; k < KX; ++k) {
    float sig2 = K.vg.fsg[k] * K.vg.fsg[k];
    float rhref = fmaxf(K.p.rhlsc + K.p.drhlsc * (sig2 - 1.0f), K.p.rhblsc);
    float dqa = rhref * qsat[k] - q[k];
    if (!found && dqa < 0.0f) {
      first = k;
      found = true;
    }
  }
  return first;
}

// RH part of the cloud-top search (shortwave_radiation.py:359-373).  Returns icltop before
// the min with iptop, and the cloud cover from relative humidity (before the precip term).
template <int KX>
__device__ __forceinline__ int cloud_rh_top(const Consts& K, const float rh[KX],
                                            const float q[KX], float& cloudc_out) {
  const spd_params_t& p = K.p;
  const int nl1 = KX - 2, nlp = KX;
  bool m0 = rh[nl1] > p.rhcl1;
  float cloudc0 = m0 ? rh[nl1] - p.rhcl1 : 0.0f;
  int icl0 = m0 ? nl1 : nlp;
  // all levels are compared against the initial cover (vectorised restatement of the loop)
  float cmax = -INFINITY;
  float upd[KX];
  int iupd[KX];
#pragma unroll
  for (int k = 2; k < KX - 2; ++k) {
    float drh = rh[k] - p.rhcl1;
    bool m = (drh > cloudc0) && (q[k] > p.qacl);
    upd[k] = m ? drh : cloudc0;
    iupd[k] = m ? k : icl0;
    cmax = fmaxf(cmax, upd[k]);
  }
  int icl = -1;
#pragma unroll
  for (int k = 2; k < KX - 2; ++k) {
    int cand = (cmax == upd[k]) ? iupd[k] : icl0;
    icl = max(icl, cand);
  }
  cloudc_out = cmax;
  return icl;
}

// Load and derive the fields the cloud-top pre-pass needs; returns icltop.
template <int KX>
__device__ __forceinline__ int column_icltop(const Consts& K, const float t[KX],
                                             const float q[KX], const float phi[KX],
                                             float psa) {
  float qsat[KX], rh[KX], se[KX];
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    qsat[k] = qsat_of(t[k], psa, K.vg.fsg[k]);
    rh[k] = q[k] / qsat[k];
    se[k] = kCp * t[k] + phi[k];
  }
  float qdif;
  int iptop = diagnose_convection<KX>(K, se, q, qsat, psa, qdif);
  iptop = min(lsc_top<KX>(K, q, qsat), iptop);
  float cl;
  int icl = cloud_rh_top<KX>(K, rh, q, cl);
  return min(iptop, icl);
}

}  // namespace spd

namespace spd {

// Per-column inputs beyond the level fields.
struct SurfaceIn {
  float psa, u_low, v_low, sst, stl, soilw, snowc, sice, alb0, fmask, orog, phis0;
};

// Per-column results.
template <int KX>
struct ColumnOut {
  float dt[KX], dq[KX];
  float du_low, dv_low;
  float precnv, precls, cbmf, cloudc, clstr, rsds, rsns, ftop_sw, rlds, rlns, ftop_lw;
  float tsfc, tskin, shf, evap;
  int iptop, icltop;
};

// The full SPEEDY physics of one column: speedy_physics.py:88-127 with the eleven terms of
// speedy_physics.py:67-80 in order, the tendencies summed in that order.  `q` is the state
// humidity after verify_state when that is fused.  `S` is the instance's cloud-top level set
// (bit l set when some column of the instance has clip(icltop, 0, kx-1) == l).
template <int KX>
__device__ __forceinline__ void column_full(const Consts& K, const float t[KX], const float q[KX],
                                            const float phi[KX], const SurfaceIn& s,
                                            const ZonalRow& z, uint32_t S, ColumnOut<KX>& o) {
  const spd_params_t& p = K.p;
  const spd_vgrid_t& vg = K.vg;
  const float psa = s.psa;
  float* dT = o.dt;
  float* dQ = o.dq;

  // ---- spec_hum_to_rel_hum (humidity.py:16-51) ----------------------------------------------
  float qsat[KX], rh[KX], se[KX];
#pragma unroll
  for (int k = 0; k < KX; ++k) {
    qsat[k] = qsat_of(t[k], psa, vg.fsg[k]);
    rh[k] = q[k] / qsat[k];
    se[k] = kCp * t[k] + phi[k];
  }

  // ---- set_forcing (physics/speedy/forcing.py:11-39) ------------------------------------------
  const float snowc = fminf(1.0f, s.snowc);
  const float alb_l = s.alb0 + snowc * (p.albsn - s.alb0);
  const float alb_s = p.albsea + s.sice * (p.albice - p.albsea);
  const float albsfc = alb_s + s.fmask * (alb_l - alb_s);
  float ablco2 = 6.0f;
  if (K.flags & SPD_INCREASE_CO2)
    ablco2 = 6.0f * expf(0.005f * ((float)K.model_year + K.tyear - (float)K.co2_year_ref));

  // ---- get_convection_tendencies (convection.py:99-237) --------------------------------------
  float qdif;
  int iptop = diagnose_convection<KX>(K, se, q, qsat, psa, qdif);
  {
    float entr[KX];
    float sentr = 0.0f;
#pragma unroll
    for (int k = 1; k < KX - 1; ++k) {
      entr[k] = sq(fmaxf(0.0f, vg.fsg[k] - 0.5f));
      sentr += entr[k];
    }
    const float escale = p.entmax / sentr;
#pragma unroll
    for (int k = 1; k < KX - 1; ++k) entr[k] = entr[k] * escale;
    const float fm0 = kP0 * vg.dhs[KX - 1] / (kGrav * p.trcnv * 3600.0f);
    const float rdps = 2.0f / (1.0f - p.psmin);
    const bool mask = iptop < KX;
    const float qmax = fmaxf(1.01f * q[KX - 1], qsat[KX - 1]);
    // half-level dry static energy / humidity, sb3[k] for k >= 1
    float sb3[KX], qb3[KX];
    sb3[0] = 0.0f;
    qb3[0] = 0.0f;
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      sb3[k] = se[k - 1] + vg.wvi[k - 1][1] * (se[k] - se[k - 1]);
      qb3[k] = q[k - 1] + vg.wvi[k - 1][1] * (q[k] - q[k - 1]);
    }
    const float sb = sb3[KX - 1];
    const float qb = fminf(qb3[KX - 1], q[KX - 1]);
    const float fpsa = psa * fminf(1.0f, (psa - p.psmin) * rdps);
    const float fmass = fm0 * fpsa * fminf(5.0f, qdif / (qmax - qb));
    const float cbmf = mask ? fmass : 0.0f * fmass;
    const float fus = fmass * se[KX - 1], fuq = fmass * qmax;
    const float fds = fmass * sb, fdq = fmass * qb;
    float dfse[KX], dfqa[KX];
    // reverse cumulative entrainment fluxes, accumulated from the surface upwards
    float cm = 0.0f, cs = 0.0f, cq = 0.0f;
    float fm3[KX], fus3[KX], fuq3[KX];
#pragma unroll
    for (int k = KX - 1; k >= 0; --k) {
      const bool lm = (k <= KX - 2) && (k >= iptop);
      float en = (k >= 1 && k <= KX - 2) ? entr[k] * psa * cbmf : 0.0f;
      en = lm ? en : 0.0f * en;
      cm = cm + en * 1.0f;
      cs = cs + en * se[k];
      cq = cq + en * q[k];
      fm3[k] = fmass + cm;
      fus3[k] = fus + cs;
      fuq3[k] = fuq + cq;
    }
    dfse[KX - 1] = fds - fus;
    dfqa[KX - 1] = fdq - fuq;
    float fsq_sum = 0.0f;
    float fsq[KX];
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      const bool lm = (k <= KX - 2) && (k >= iptop);
      if (k < KX - 1) {
        const float fds_k1 = (k + 1 == KX - 1) ? fds : fm3[k + 1] * sb3[k + 1];
        const float fdq_k1 = (k + 1 == KX - 1) ? fdq : fm3[k + 1] * qb3[k + 1];
        const float a = (fus3[k + 1] - fds_k1) - (fus3[k] - fm3[k] * sb3[k]);
        const float b = (fuq3[k + 1] - fdq_k1) - (fuq3[k] - fm3[k] * qb3[k]);
        dfse[k] = lm ? a : 0.0f * a;
        dfqa[k] = lm ? b : 0.0f * b;
      }
      const float delq = lm ? (p.rhil * qsat[k] - q[k]) : 0.0f * (p.rhil * qsat[k] - q[k]);
      fsq[k] = (delq > 0.0f ? p.smf : 0.0f * p.smf) * cbmf * delq;
    }
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      dfqa[k] = dfqa[k] + fsq[k];
      fsq_sum += fsq[k];
    }
    dfqa[KX - 1] = dfqa[KX - 1] + (-fsq_sum);
    // top layer: condensation and detrainment at k = iptop - 1 (dropped when iptop - 1 >= kx)
    float precnv = 0.0f;
    if (iptop <= KX - 1) {
      const int it = iptop;  // 3 .. kx-3 when convecting
      float fm_t = 0.f, fus_t = 0.f, fuq_t = 0.f, fds_t = 0.f, fdq_t = 0.f, qsatb = 0.f;
#pragma unroll
      for (int k = 0; k < KX; ++k) {
        if (k == it) {
          fm_t = fm3[k];
          fus_t = fus3[k];
          fuq_t = fuq3[k];
          fds_t = (k == KX - 1) ? fds : fm3[k] * sb3[k];
          fdq_t = (k == KX - 1) ? fdq : fm3[k] * qb3[k];
        }
        if (k == it - 1 && k < KX - 1)
          qsatb = qsat[k] + vg.wvi[k][1] * (qsat[k + 1] - qsat[k]);
      }
      precnv = fmaxf(fuq_t - fm_t * qsatb, 0.0f);
#pragma unroll
      for (int k = 0; k < KX; ++k) {
        if (k == it - 1) {
          dfse[k] = fus_t - fds_t + kAlhc * precnv;
          dfqa[k] = fuq_t - fdq_t - precnv;
        }
      }
    } else {
      // iptop == kx+1: the padded gathers read zeros, precnv = max(0 - 0*0, 0)
      precnv = 0.0f;
    }
    const float rps = 1.0f / psa;
    dT[0] = dfse[0];
    dQ[0] = dfqa[0];
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      dT[k] = dfse[k] * rps * vg.grdscp[k];
      dQ[k] = dfqa[k] * rps * vg.grdsig[k];
    }
    o.cbmf = cbmf;
    o.precnv = precnv;
  }

  // ---- get_large_scale_condensation_tendencies (large_scale_condensation.py:14-86) ----------
  {
    const float rtlsc = 1.0f / (p.trlsc * 3600.0f);
    const float tfact = (float)(2501.0 / 1004.0);
    const float prg = (float)(1e5 / 9.81);
    const float psa2 = psa * psa;
    float psum = 0.0f;
    int first = 1;
    bool found = false;
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      const float sig2 = vg.fsg[k] * vg.fsg[k];
      const float rhref = fmaxf(p.rhlsc + p.drhlsc * (sig2 - 1.0f), p.rhblsc);
      const float dqmax = 10.0f * sig2 * rtlsc;
      const float dqa = rhref * qsat[k] - q[k];
      float dql = 0.0f, dtl = 0.0f;
      if (dqa < 0.0f) {
        dql = dqa * rtlsc;
        dtl = tfact * fminf(-dql, dqmax * psa2);
        if (!found) {
          first = k;
          found = true;
        }
      }
      dT[k] = dT[k] + dtl;
      dQ[k] = dQ[k] + dql;
      psum += (vg.dhs[k] * prg) * dql;
    }
    o.precls = (0.0f - psum) * psa;
    iptop = min(first, iptop);
  }
  o.iptop = iptop;

  // ---- get_clouds / clouds (shortwave_radiation.py:298-404) ---------------------------------
  float cloudc, clstr, qcloud;
  int icltop;
  {
    float cl;
    int icl = cloud_rh_top<KX>(K, rh, q, cl);
    const float gse = (se[KX - 2] - se[KX - 1]) / (phi[KX - 2] - phi[KX - 1]);
    const float rrcl = 1.0f / (p.rhcl2 - p.rhcl1);
    const float pr1 = fminf(p.pmaxcl, 86.4f * (o.precnv + o.precls));
    cloudc = fminf(1.0f, p.wpcl * sqrtf(fmaxf(kEpsilon, pr1)) + sq(fminf(1.0f, cl * rrcl)));
    if (isnan(cloudc)) cloudc = 1.0f;
    icltop = min(iptop, icl);
    qcloud = q[KX - 2];
    const float rgse = 1.0f / (p.gse_s1 - p.gse_s0);
    const float fstab = fminf(fmaxf(rgse * (gse - p.gse_s0), 0.0f), 1.0f);
    clstr = fstab * fmaxf(p.clsmax - 1.2f * cloudc, 0.0f);
    const float clstrl = fmaxf(clstr, p.clsminl) * rh[KX - 1];
    clstr = clstr + s.fmask * (clstrl - clstr);
  }
  o.cloudc = cloudc;
  o.clstr = clstr;
  o.icltop = icltop;

  // ---- get_shortwave_rad_fluxes (shortwave_radiation.py:12-217) -----------------------------
  float flux_sw0, flux_sw1;  // mod_radcon.flux bands 0 and 1 handed to the LW upward pass
  float rsds;
  {
    const float fband2 = 0.05f, fband1 = 0.95f;
    const bool cmask = icltop < KX;
    const float refl = cmask ? p.albcl * cloudc : 0.0f;
    float tau0[KX], r[KX], dfabs[KX];
    const float psaz = psa * z.zenit;
    const float acloud = cloudc * fminf(p.abscl1 * qcloud, p.abscl2);
#pragma unroll
    for (int k = 0; k < KX; ++k) r[k] = ((S >> k) & 1u) ? refl : 0.0f;
    r[KX - 1] = p.albcls * clstr;
    tau0[0] = expf(-psaz * vg.dhs[0] * p.absdry);
#pragma unroll
    for (int k = 1; k < KX - 1; ++k) {
      const float abs1 = p.absdry + p.absaer * (vg.fsg[k] * vg.fsg[k]);
      const float cl = (k >= icltop) ? acloud : 0.0f;
      tau0[k] = expf(-psaz * vg.dhs[k] * (abs1 + p.abswv1 * q[k] + cl));
    }
    {
      const float abs1 = p.absdry + p.absaer * (vg.fsg[KX - 1] * vg.fsg[KX - 1]);
      tau0[KX - 1] = expf(-psaz * vg.dhs[KX - 1] * (abs1 + p.abswv1 * q[KX - 1]));
    }
    // downward, band 1
    float f1 = z.fsol * fband1;
    dfabs[0] = f1;
    f1 = tau0[0] * (f1 - z.ozupp * psa);
    dfabs[0] = dfabs[0] + (-f1);
    dfabs[1] = f1;
    f1 = tau0[1] * (f1 - z.ozone * psa);
    dfabs[1] = dfabs[1] + (-f1);
#pragma unroll
    for (int k = 2; k < KX; ++k) {
      const float prev = f1;
      f1 = prev * tau0[k] * (1.0f - r[k]);
      dfabs[k] = prev * (1.0f - r[k]) * (1.0f - tau0[k]);
      r[k] = r[k] * prev;
    }
    // downward, band 2
    float f2 = z.fsol * fband2;
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      const float tau1 = expf(-psaz * vg.dhs[k] * p.abswv2 * q[k]);
      const float prev = f2;
      f2 = prev * tau1;
      dfabs[k] = dfabs[k] + prev * (1.0f - tau1);
    }
    // surface reflection and upward pass
    rsds = f1 + f2;
    float up = f1 * albsfc;
    o.rsns = rsds - up;
    dfabs[KX - 1] = dfabs[KX - 1] + up * (1.0f - tau0[KX - 1]);
#pragma unroll
    for (int k = KX - 1; k >= 1; --k) {
      up = up * tau0[k] + r[k];
      dfabs[k - 1] = dfabs[k - 1] + up * (1.0f - tau0[k - 1]);
    }
    const float ftop_up = tau0[0] * up + r[0];
    o.ftop_sw = z.fsol - ftop_up;
    flux_sw0 = ftop_up;
    flux_sw1 = f2;
    const bool gate = (K.model_step % 3) == 0;
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      const float tsw = dfabs[k] * vg.grdscp[k] / psa;
      dT[k] = dT[k] + (gate ? tsw : 0.0f);
    }
  }
  o.rsds = rsds;

  // ---- longwave transmissivities (shortwave_radiation.py:174-206) ---------------------------
  // tau_lw(k, b) is recomputed where it is used, from these per-column constants.
  const float acl1 = cloudc * p.ablcl1, acl2 = cloudc * p.ablcl2;
  auto lw_tau = [&](int k, float tau[4]) {
    float a0 = p.ablwin, a1 = ablco2, a2 = p.ablwv1 * q[k], a3 = p.ablwv2 * q[k];
    if (k == 0) {
      a2 = 0.0f;
      a3 = 0.0f;
    }
    if (k >= 2 && k <= KX - 2) {
      a0 = a0 + ((k > icltop) ? acl1 : acl2);
      a2 = fmaxf(a2, acl2);
      a3 = fmaxf(a3, acl2);
    }
    tau[0] = expf(-a0 * psa * vg.dhs[k]);
    tau[1] = expf(-a1 * psa * vg.dhs[k]);
    tau[2] = expf(-a2 * psa * vg.dhs[k]);
    tau[3] = expf(-a3 * psa * vg.dhs[k]);
  };
  const float eps1 = p.epslw / (vg.dhs[0] + vg.dhs[1]);
  const float stratc0 = z.stratz * psa, stratc1 = eps1 * psa;

  // ---- blackbody emission st4a (longwave_radiation.py:42-68) --------------------------------
  float st0[KX], st1[KX];
  {
    float th[KX];
#pragma unroll
    for (int k = 0; k < KX - 1; ++k) th[k] = t[k] + vg.wvi[k][1] * (t[k + 1] - t[k]);
    const float s10 = 0.75f * t[0] + 0.25f * th[0];
    const float s11 = 0.50f * t[1] + 0.25f * (th[0] + th[1]);
    st0[0] = kSbc * (sq(s10) * sq(s10));
    st1[0] = 0.0f;
    st0[1] = kSbc * (sq(s11) * sq(s11));
    st1[1] = 0.0f;
#pragma unroll
    for (int k = 2; k < KX; ++k) {
      const float grad = (k < KX - 1) ? 0.5f * fmaxf(th[k] - th[k - 1], 0.0f)
                                      : fmaxf(t[KX - 1] - th[KX - 2], 0.0f);
      const float st3 = kSbc * (t[k] * t[k] * t[k]);
      st0[k] = st3 * t[k];
      st1[k] = 4.0f * st3 * grad;
    }
  }

  // ---- get_downward_longwave_rad_fluxes (longwave_radiation.py:13-117) ----------------------
  float dfl[KX];
  float rlds;
  {
    float fl[4], tau[4], fb[4];
    lw_tau(0, tau);
    radset(t[0], p.epslw, fb);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float emis = 1.0f - tau[b];
      fl[b] = emis * (fb[b] * (st0[0] + emis * st1[0]));
    }
    fl[2] = 0.0f;
    fl[3] = 0.0f;
    float sprev = sum4(fl);
    dfl[0] = 0.0f + (-sprev);
#pragma unroll
    for (int k = 1; k < KX; ++k) {
      lw_tau(k, tau);
      radset(t[k], p.epslw, fb);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const float emis = 1.0f - tau[b];
        fl[b] = tau[b] * fl[b] + emis * (fb[b] * (st0[k] + emis * st1[k]));
      }
      const float sk = sum4(fl);
      dfl[k] = 0.0f + (-(sk - sprev));
      sprev = sk;
    }
    const float ef[4] = {p.emisfc * fl[0], p.emisfc * fl[1], p.emisfc * fl[2], p.emisfc * fl[3]};
    rlds = sum4(ef);
    const float corlw = p.epslw * p.emisfc * st0[KX - 1];
    dfl[KX - 1] = dfl[KX - 1] + (-corlw);
    rlds = rlds + corlw;
  }
  o.rlds = rlds;

  // ---- get_surface_fluxes (surface_flux.py:15-300) ------------------------------------------
  float rlus2 = 0.0f, tsfc = 0.0f, tskin_out = 0.0f;
  {
    const float esbc = p.emisfc * kSbc;
    const float ghum0 = 1.0f - p.fhum0;
    const float ta1 = t[KX - 1], ta2 = t[KX - 2];
    const float ua = s.u_low, va = s.v_low;
    const float phi0 = s.orog * kGrav;
    const float u0 = p.fwind0 * ua, v0 = p.fwind0 * va;
    float ustr0 = 0.f, ustr1 = 0.f, vstr0 = 0.f, vstr1 = 0.f, shf0 = 0.f, shf1 = 0.f;
    float evap0 = 0.f, evap1 = 0.f, rlus0 = 0.f, rlus1 = 0.f;
    float t1_1 = 0.f, q1_1 = 0.f, denv2 = 0.f, tskin = 0.f;
    const float astab = (K.flags & SPD_LSCASYM) ? 0.5f : 1.0f;
    const float rdth = p.fstab / p.dtheta;
    const bool land = (K.flags & SPD_LFLUXLAND) != 0;
    if (land) {
      const float rcp = (float)(1.0 / 1004.0);
      const float gtemp0 = 1.0f - p.ftemp0;
      const float dt1 = vg.wvi[KX - 1][1] * (ta1 - ta2);
      float t1_0 = 0.0f + (ta1 + dt1);
      t1_1 = t1_0 - phi0 * dt1 / ((float)(kRgasD * 288.0) * vg.sigl[KX - 1]);
      const float t2_1 = ta1 + rcp * phi[KX - 1];
      const float t2_0 = t2_1 - rcp * phi0;
      if (ta1 > ta2) {
        t1_0 = p.ftemp0 * t1_0 + gtemp0 * t2_0;
        t1_1 = p.ftemp0 * t1_1 + gtemp0 * t2_1;
      } else {
        t1_0 = ta1;
        t1_1 = ta1;
      }
      const float t0 = t1_1 + s.fmask * (t1_0 - t1_1);
      const float denv0 = (kP0 * psa / (kRgas * t0)) * sqrtf(u0 * u0 + v0 * v0 + p.vgust * p.vgust);
      tskin = s.stl + p.ctday * z.sqrt_coa * rsds * (1.0f - alb_l) * psa;
      const float dthl = (tskin > t2_0) ? fminf(p.dtheta, tskin - t2_0)
                                        : fmaxf(-p.dtheta, astab * (tskin - t2_0));
      const float denv1 = denv0 * (1.0f + dthl * rdth);
      const float rhdrag = 1.0f / (kGrav * p.hdrag);
      const float forog = 1.0f + rhdrag * (1.0f - expf(-fmaxf(s.phis0, 0.0f) * rhdrag));
      const float cdldv = p.cdl * denv0 * forog;
      ustr0 = -cdldv * ua;
      vstr0 = -cdldv * va;
      const float chlcp = p.chl * kCp;
      shf0 = chlcp * denv1 * (tskin - t1_0);
      float q1_0;
      if (p.fhum0 > 0.0f) {
        q1_0 = p.fhum0 * (rh[KX - 1] * qsat_of(t1_0, psa, 1.0f)) + ghum0 * q[KX - 1];
      } else {
        q1_0 = q[KX - 1];
      }
      const float qs00 = qsat_of(tskin, psa, 1.0f);
      evap0 = p.chl * denv1 * fmaxf(0.0f, s.soilw * qs00 - q1_0);
      const float tsk3 = tskin * tskin * tskin;
      const float drls = 4.0f * esbc * tsk3;
      rlus0 = esbc * tsk3 * tskin;
      float hfl0 = rsds * (1.0f - alb_l) + rlds - (rlus0 + shf0 + (kAlhc * evap0));
      if (K.flags & SPD_LSKINEB) {
        const float clamb = p.clambda + (snowc * (p.clambsn - p.clambda));
        hfl0 = hfl0 - (clamb * (tskin - s.stl));
        float qs01 = qsat_of(tskin + 1.0f, psa, 1.0f);
        qs01 = (evap0 > 0.0f) ? s.soilw * (qs01 - qs00) : 0.0f;
        const float dtskin =
            hfl0 / (clamb + drls + (p.chl * denv1 * (kCp + (kAlhc * qs01))));
        tskin = tskin + dtskin;
        shf0 = shf0 + chlcp * denv1 * dtskin;
        evap0 = evap0 + p.chl * denv1 * qs01 * dtskin;
        rlus0 = rlus0 + drls * dtskin;
      }
      const float sst = s.sst;
      const float dths = (sst > t2_1) ? fminf(p.dtheta, sst - t2_1)
                                      : fmaxf(-p.dtheta, astab * (sst - t2_1));
      denv2 = denv0 * (1.0f + dths * rdth);
      if (p.fhum0 > 0.0f) {
        q1_1 = p.fhum0 * (rh[KX - 1] * qsat_of(t1_1, psa, 1.0f)) + ghum0 * q[KX - 1];
      } else {
        q1_1 = q[KX - 1];
      }
      const float cdsdv = p.cds * denv2;
      ustr1 = -cdsdv * ua;
      vstr1 = -cdsdv * va;
    }
    // sea
    const float sst = s.sst;
    shf1 = p.chs * kCp * denv2 * (sst - t1_1);
    const float qs1 = qsat_of(sst, psa, 1.0f);
    evap1 = p.chs * denv2 * (qs1 - q1_1);
    rlus1 = esbc * (sq(sst) * sq(sst));
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
    const float rps = 1.0f / psa;
    o.du_low = 0.0f + ustr2 * rps * vg.grdsig[KX - 1];
    o.dv_low = 0.0f + vstr2 * rps * vg.grdsig[KX - 1];
    dT[KX - 1] = dT[KX - 1] + (0.0f + shf2 * rps * vg.grdscp[KX - 1]);
    dQ[KX - 1] = dQ[KX - 1] + (0.0f + evap2 * rps * vg.grdsig[KX - 1]);
    o.shf = shf2;
    o.evap = evap2;
  }
  o.tsfc = tsfc;
  o.tskin = tskin_out;

  // ---- get_upward_longwave_rad_fluxes (longwave_radiation.py:119-202) -----------------------
  {
    const float refsfc = 1.0f - p.emisfc;
    o.rlns = rlus2 - rlds;
    float fb[4], fl[4], tau[4];
    radset(tsfc, p.epslw, fb);
    const float fsw[4] = {flux_sw0, flux_sw1, 0.0f, 0.0f};
#pragma unroll
    for (int b = 0; b < 4; ++b) fl[b] = fb[b] * rlus2 + refsfc * fsw[b];
    dfl[KX - 1] = dfl[KX - 1] + p.epslw * rlus2;
    float sk = sum4(fl);
#pragma unroll
    for (int k = KX - 1; k >= 1; --k) {
      lw_tau(k, tau);
      radset(t[k], p.epslw, fb);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const float emis = 1.0f - tau[b];
        fl[b] = tau[b] * fl[b] + emis * (fb[b] * (st0[k] - emis * st1[k]));
      }
      const float skm1 = sum4(fl);
      dfl[k] = dfl[k] + (sk - skm1);
      sk = skm1;
    }
    lw_tau(0, tau);
    radset(t[0], p.epslw, fb);
    float top[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float emis = 1.0f - tau[b];
      top[b] = (b < 2) ? tau[b] * fl[b] + emis * (fb[b] * (st0[0] - emis * st1[0])) : fl[b];
    }
    dfl[0] = dfl[0] + ((fl[0] - top[0]) + (fl[1] - top[1]));
    const float corlw1 = vg.dhs[0] * stratc1 * st0[0] + stratc0;
    const float corlw2 = vg.dhs[1] * stratc1 * st0[1];
    dfl[0] = dfl[0] + (-corlw1);
    dfl[1] = dfl[1] + (-corlw2);
    o.ftop_lw = (corlw1 + corlw2) + sum4(top);
#pragma unroll
    for (int k = 0; k < KX; ++k) dT[k] = dT[k] + dfl[k] * vg.grdscp[k] / psa;
  }

  // ---- get_vertical_diffusion_tend (vertical_diffusion.py:10-136) ---------------------------
  {
    const spd_params_t& pv = p;
    const int nl1 = KX - 1;
    const int icnv = KX - iptop - 1;
    const float cshc = vg.dhs[KX - 1] / 3600.0f;
    const float cvdi = (vg.hsg[nl1] - vg.hsg[1]) / ((float)(nl1 - 1) * 3600.0f);
    const float fshcq = cshc / pv.trshc;
    const float fshcse = cshc / (pv.trshc * kCp);
    const float fvdiq = cvdi / pv.trvdi;
    const float fvdise = cvdi / (pv.trvds * kCp);
    float tt[KX], qt[KX];
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      tt[k] = 0.0f;
      qt[k] = 0.0f;
    }
    const float drh0 = pv.rhgrad * (vg.fsg[KX - 1] - vg.fsg[nl1 - 1]);
    const float fvdiq2 = fvdiq * vg.hsg[nl1];
    const float dmse = se[KX - 1] - se[nl1 - 1] + kAlhc * (q[KX - 1] - qsat[nl1 - 1]);
    const float drh = rh[KX - 1] - rh[nl1 - 1];
    const float fcnv = (icnv > 0 && dmse >= 0.0f) ? pv.redshc : 1.0f;
    if (dmse >= 0.0f) {
      const float fluxse = fcnv * fshcse * dmse;
      tt[nl1 - 1] = fluxse * (1.0f / vg.dhs[nl1 - 1]);
      tt[KX - 1] = -fluxse * (1.0f / vg.dhs[KX - 1]);
      if (drh >= 0.0f) {
        const float fq = fcnv * fshcq * qsat[KX - 1] * drh;
        qt[nl1 - 1] = fq * (1.0f / vg.dhs[nl1 - 1]);
        qt[KX - 1] = -fq * (1.0f / vg.dhs[KX - 1]);
      }
    } else if (dmse < 0.0f && drh > drh0) {
      const float fq = fvdiq2 * qsat[nl1 - 1] * drh;
      qt[nl1 - 1] = fq * (1.0f / vg.dhs[nl1 - 1]);
      qt[KX - 1] = -fq * (1.0f / vg.dhs[KX - 1]);
    }
    // moisture diffusion above the PBL: all "+" updates first, then all "-" updates
    float fluxq[KX];
#pragma unroll
    for (int k = 2; k < KX - 2; ++k) {
      const bool cond = vg.hsg[k + 1] > 0.5f;
      const float d0 = pv.rhgrad * (vg.fsg[k + 1] - vg.fsg[k]);
      const float f2 = fvdiq * vg.hsg[k + 1];
      const float dr = rh[k + 1] - rh[k];
      fluxq[k] = (dr >= d0 && cond) ? f2 * qsat[k] * dr : 0.0f;
      qt[k] = qt[k] + fluxq[k] * (1.0f / vg.dhs[k]);
    }
#pragma unroll
    for (int k = 2; k < KX - 2; ++k) qt[k + 1] = qt[k + 1] + (-fluxq[k] * (1.0f / vg.dhs[k + 1]));
    // damping of super-adiabatic lapse rate
    // all "+fluxse*rsig" updates first, then the cumulative compensation
    float fse[KX];
#pragma unroll
    for (int k = 0; k < nl1; ++k) {
      const float se0 = se[k + 1] - pv.segrad * (phi[k + 1] - phi[k]);
      fse[k] = (se[k] < se0) ? fvdise * (se0 - se[k]) : 0.0f;
      tt[k] = tt[k] + fse[k] * (1.0f / vg.dhs[k]);
    }
    float cum = 0.0f;
#pragma unroll
    for (int k = 0; k < nl1; ++k) {
      cum = cum + fse[k] * (1.0f / (1.0f - vg.hsg[k + 1]));
      tt[k + 1] = tt[k + 1] + (-cum);
    }
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      dT[k] = dT[k] + tt[k];
      dQ[k] = dQ[k] + qt[k];
    }
  }
}

}  // namespace spd
