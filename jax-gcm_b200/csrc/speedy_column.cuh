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
// Stages of the adjoint's cloud-top pre-pass (the level set S from registers).
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

}  // namespace spd
